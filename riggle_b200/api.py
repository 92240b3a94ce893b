"""Python face of the C ABI, named after the reference crate's types and functions.

`LayerConfig` mirrors src/io/meta.rs:23-90; `Index` is the device-resident form of the database a
query opens (src/tasks/query/mod.rs:124-233); `Context.query_counts` replaces the counting sweep of
query_database (src/tasks/query/mod.rs:182-307) and returns the dense count matrix together with
exact overlap base pairs.  All compute happens in libriggle_b200.so on the GPU.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, load


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else None


class LayerConfig:
    """LayerConfig (src/io/meta.rs:23-90)."""

    def __init__(self, min_size=128, growth_factor=4):
        self.min_size = int(min_size)
        self.growth_factor = int(growth_factor)

    @classmethod
    def default_genomic(cls):
        return cls(128, 4)

    def layer_for_size(self, size):
        return load().rgl_layer_for_size(self.min_size, self.growth_factor, int(size))

    def layer_max_size(self, layer):
        return load().rgl_layer_max_size(self.min_size, self.growth_factor, int(layer))

    def tile_size(self, layer):
        return load().rgl_tile_size(self.min_size, self.growth_factor, int(layer))


class Index:
    """A database index resident in HBM (the handle owns the device memory)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        info = _lib.IndexInfo()
        check(load().rgl_index_get_info(self._h, C.byref(info)))
        self.num_sources = info.num_sources
        self.num_shards = info.num_shards
        self.num_layer_slots = info.num_layer_slots
        self.num_layers = info.num_layers
        self.num_intervals = info.num_intervals
        self.device_bytes = info.device_bytes
        self.device = info.device

    @classmethod
    def open(cls, db_dir, device=0):
        """Opens a database directory written by the reference's `add`."""
        h = C.c_void_p()
        check(load().rgl_index_open(str(db_dir).encode(), device, C.byref(h)))
        return cls(h)

    @classmethod
    def from_layers(cls, layers, num_sources, shard_names, min_size=128, growth_factor=4, source_names=None,
                    device=0):
        """layers: {(shard_id, layer): (pos uint32[n,2] sorted by start, sid uint32[n])}."""
        keep = []
        descs = (_lib.LayerDesc * max(1, len(layers)))()
        for i, ((sh, k), (pos, sid)) in enumerate(sorted(layers.items())):
            pos = np.ascontiguousarray(pos, dtype=np.uint32).reshape(-1, 2)
            sid = np.ascontiguousarray(sid, dtype=np.uint32).reshape(-1)
            keep += [pos, sid]
            descs[i] = _lib.LayerDesc(int(sh), int(k), len(sid), _ptr(pos), _ptr(sid))
        names = (C.c_char_p * max(1, len(shard_names)))(*[s.encode() for s in shard_names])
        srcs = None
        if source_names is not None:
            srcs = (C.c_char_p * max(1, len(source_names)))(*[s.encode() for s in source_names])
        d = _lib.IndexDesc(min_size, growth_factor, num_sources, len(shard_names), names, srcs, len(layers), descs)
        h = C.c_void_p()
        check(load().rgl_index_open_mem(C.byref(d), device, C.byref(h)))
        return cls(h)

    @classmethod
    def synth(cls, spec, min_size=128, growth_factor=4, device=0):
        """Builds a seeded synthetic database directly in HBM (see SynthSpec)."""
        h = C.c_void_p()
        check(load().rgl_index_synth(C.byref(spec.c), min_size, growth_factor, device, C.byref(h)))
        return cls(h)

    @classmethod
    def synth_columns(cls, spec, file_lo, file_hi, min_size=128, growth_factor=4, device=0):
        """Files [file_lo, file_hi) of a synthetic database (a column shard), sids rebased to 0."""
        h = C.c_void_p()
        check(load().rgl_index_synth_columns(C.byref(spec.c), min_size, growth_factor, file_lo, file_hi, device,
                                             C.byref(h)))
        return cls(h)

    @classmethod
    def from_beds(cls, input_path, min_size=128, growth_factor=4, threads=0, device=0):
        """add_to_database into a new device index from the BED files of a directory (or one file)."""
        h = C.c_void_p()
        check(load().rgl_index_add_beds(None, str(input_path).encode(), min_size, growth_factor, threads, device,
                                        C.byref(h)))
        return cls(h)

    def add_beds(self, input_path, threads=0):
        """A new index: this one with the BED files of input_path merged in (next D_SIDs)."""
        h = C.c_void_p()
        check(load().rgl_index_add_beds(self._h, str(input_path).encode(), 0, 0, threads, self.device, C.byref(h)))
        return Index(h)

    def write(self, db_dir):
        """Writes the reference's database layout (meta.json, shards/<shard>/layer_K.{pos,sid,idx})."""
        check(load().rgl_index_write(self._h, str(db_dir).encode()))

    def select_columns(self, sid_lo, sid_hi):
        """A new index holding sources [sid_lo, sid_hi) of this one (sids rebased to 0)."""
        h = C.c_void_p()
        check(load().rgl_index_select_columns(self._h, sid_lo, sid_hi, C.byref(h)))
        return Index(h)

    def shard_id(self, name):
        out = C.c_uint32()
        check(load().rgl_index_shard_id(self._h, name.encode(), C.byref(out)))
        return out.value

    def shard_name(self, shard):
        r = load().rgl_index_shard_name(self._h, shard)
        return r.decode() if r else None

    def source_name(self, sid):
        r = load().rgl_index_source_name(self._h, sid)
        return r.decode() if r else None

    def layer_count(self, shard, layer):
        return load().rgl_index_layer_count(self._h, shard, layer)

    def export_layer(self, shard, layer):
        n = self.layer_count(shard, layer)
        pos = np.empty((n, 2), np.uint32)
        sid = np.empty(n, np.uint32)
        if n:
            check(load().rgl_index_export_layer(self._h, shard, layer, _ptr(pos), _ptr(sid)))
        return pos, sid

    def close(self):
        if self._h:
            load().rgl_index_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA stream + reusable device workspace bound to an Index."""

    def __init__(self, index, stream=None):
        self.index = index
        h = C.c_void_p()
        check(load().rgl_context_create(index._h, C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h

    @property
    def stream(self):
        return load().rgl_context_stream(self._h)

    def reserve(self, max_intervals, max_rows):
        check(load().rgl_context_reserve(self._h, int(max_intervals), int(max_rows)))

    def sync(self):
        check(load().rgl_context_sync(self._h))

    @staticmethod
    def _opts(chunk=0, ctas_per_sm=0, counts_only=False, pair_ratio=0):
        return _lib.QueryOpts(chunk, ctas_per_sm, 0, 1 if counts_only else 0, pair_ratio)

    def query_counts(self, shards, num_rows, with_overlap=True, chunk=0, ctas_per_sm=0, out=None, pair_ratio=0):
        """shards: {shard name (str) or id (int): uint32[n,3] (start, end, row)}.

        Returns (counts uint32[num_rows, D], overlap_bp uint64[num_rows, D] or None, stats dict).
        """
        keep = []
        batch = self._batch(shards, num_rows, keep)
        D = self.index.num_sources
        if out is None:
            counts = np.empty((num_rows, D), np.uint32)
            bp = np.empty((num_rows, D), np.uint64) if with_overlap else None
        else:
            counts, bp = out
        st = _lib.QueryStats()
        opts = self._opts(chunk, ctas_per_sm, not with_overlap, pair_ratio)
        check(load().rgl_query_counts(self._h, C.byref(batch), C.byref(opts), _ptr(counts), _ptr(bp), C.byref(st)))
        return counts, bp, st.as_dict()

    @staticmethod
    def _batch(shards, num_rows, keep):
        arr = (_lib.QueryShard * max(1, len(shards)))()
        for i, (k, ivs) in enumerate(shards.items()):
            ivs = np.ascontiguousarray(ivs, dtype=np.uint32).reshape(-1, 3)
            keep.append(ivs)
            if isinstance(k, str):
                arr[i] = _lib.QueryShard(k.encode(), 0, len(ivs), _ptr(ivs))
            else:
                arr[i] = _lib.QueryShard(None, int(k), len(ivs), _ptr(ivs))
        keep.append(arr)
        return _lib.QueryBatch(int(num_rows), len(shards), arr)

    def query_pairs(self, shards, num_rows):
        """`--intervals` mode: every overlapping pair as uint32[n, 8] records (query_start, query_end,
        db_start, db_end, row, sid, shard, intersection_bp)."""
        keep = []
        batch = self._batch(shards, num_rows, keep)
        n = C.c_uint64()
        check(load().rgl_query_pairs(self._h, C.byref(batch), 0, None, C.byref(n)))
        out = np.empty((n.value, 8), np.uint32)
        if n.value:
            check(load().rgl_query_pairs(self._h, C.byref(batch), n.value, _ptr(out), C.byref(n)))
        return out

    def query_batch_device(self, batch, d_counts, d_bp=None, graph=False, tuned=False, sub_batch=0, chunk=0,
                           ctas_per_sm=0, pair_ratio=0, counts_only=False, stats=True, region_bits=0,
                           global_tally=False):
        """Batched form over a DeviceBatch; d_counts / d_bp are device pointers (int) to num_rows x D
        uint32 / uint64.  Returns the stats dict (synchronising) or None (asynchronous)."""
        flags = (_lib.RGL_BF_GRAPH if graph else 0) | (_lib.RGL_BF_TUNED if tuned else 0)
        q = self._opts(chunk, ctas_per_sm, counts_only, pair_ratio)
        if global_tally:
            q.flags |= _lib.RGL_QF_GLOBAL_TALLY
        o = _lib.BatchOpts(q, int(sub_batch), flags, int(region_bits))
        st = _lib.BatchStats() if stats else None
        check(load().rgl_query_batch_device(self._h, C.byref(batch.c), C.byref(o), C.c_void_p(d_counts),
                                            C.c_void_p(d_bp) if d_bp else None, C.byref(st) if stats else None))
        return st.as_dict() if stats else None

    def query_batch_host(self, batch, h_intervals, with_overlap=True, tuned=False, sub_batch=0, chunk=0,
                         ctas_per_sm=0, pair_ratio=0, out=None, region_bits=0):
        """Batched form with host intervals (uint32[n,3] array or an int pointer to pinned memory);
        returns (counts uint32[R, D], overlap_bp uint64[R, D] or None, stats dict)."""
        R, D = batch.num_rows, self.index.num_sources
        if out is None:
            counts = np.empty((R, D), np.uint32)
            bp = np.empty((R, D), np.uint64) if with_overlap else None
        else:
            counts, bp = out
        if isinstance(h_intervals, np.ndarray):
            h = np.ascontiguousarray(h_intervals, np.uint32)
            hp = _ptr(h)
        else:
            hp = C.c_void_p(int(h_intervals))
        flags = _lib.RGL_BF_TUNED if tuned else 0
        o = _lib.BatchOpts(self._opts(chunk, ctas_per_sm, not with_overlap, pair_ratio), int(sub_batch), flags,
                           int(region_bits))
        st = _lib.BatchStats()
        check(load().rgl_query_batch_host(self._h, C.byref(batch.c), hp, C.byref(o), _ptr(counts), _ptr(bp),
                                          C.byref(st)))
        return counts, bp, st.as_dict()

    def autotune(self, batch, sub_batch=0, max_trials=64):
        """Runs the launch-shape autotuner on the batch; returns (best opts dict, list of trials)."""
        best = _lib.QueryOpts()
        trials = (_lib.TuneTrial * max_trials)()
        nt = C.c_uint32()
        check(load().rgl_batch_autotune(self._h, C.byref(batch.c), int(sub_batch), C.byref(best), trials, max_trials,
                                        C.byref(nt)))
        out = [dict(chunk=t.chunk, ctas_per_sm=t.ctas_per_sm, pair_ratio=t.pair_ratio, sweep_ms=t.sweep_ms)
               for t in trials[:min(nt.value, max_trials)]]
        return dict(chunk=best.chunk, ctas_per_sm=best.ctas_per_sm, pair_ratio=best.pair_ratio), out

    def check(self):
        check(load().rgl_context_check(self._h))

    def close(self):
        if self._h:
            load().rgl_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BedBatch:
    """Parsed BED query files (rgl_bed_batch): rows = non-empty files in path order."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, query_path, threads=0):
        """parse_file_batch over the *.bed / *.bed.gz files of a directory (or one file)."""
        h = C.c_void_p()
        check(load().rgl_bed_batch_load(str(query_path).encode(), threads, C.byref(h)))
        return cls(h)

    @classmethod
    def parse_string(cls, text, sid=0):
        data = text.encode() if isinstance(text, str) else bytes(text)
        h = C.c_void_p()
        check(load().rgl_bed_parse_string(data, len(data), sid, C.byref(h)))
        return cls(h)

    @property
    def rows(self):
        return load().rgl_bed_batch_rows(self._h)

    def name(self, row):
        r = load().rgl_bed_batch_row_name(self._h, row)
        return r.decode() if r is not None else None

    def count(self, row):
        return load().rgl_bed_batch_row_count(self._h, row)

    def shards(self, row):
        """{shard name: uint32[n,3] (start, end, sid)} of one row, in first-appearance order."""
        out = {}
        for k in range(load().rgl_bed_batch_row_shards(self._h, row)):
            name, ptr, n = C.c_char_p(), C.c_void_p(), C.c_uint64()
            check(load().rgl_bed_batch_block(self._h, row, k, C.byref(name), C.byref(ptr), C.byref(n)))
            a = np.ctypeslib.as_array((C.c_uint32 * (3 * n.value)).from_address(ptr.value)).reshape(-1, 3).copy() \
                if n.value else np.zeros((0, 3), np.uint32)
            out[name.value.decode()] = a
        return out

    def query(self, ctx, with_overlap=True):
        """Counting path of query_database over the batch: (counts, overlap_bp, stats)."""
        D = ctx.index.num_sources
        counts = np.empty((self.rows, D), np.uint32)
        bp = np.empty((self.rows, D), np.uint64) if with_overlap else None
        st = _lib.QueryStats()
        opts = Context._opts(counts_only=not with_overlap)
        check(load().rgl_bed_batch_query(ctx._h, self._h, C.byref(opts), _ptr(counts), _ptr(bp), C.byref(st)))
        return counts, bp, st.as_dict()

    def close(self):
        if self._h:
            load().rgl_bed_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request server over a resident Index (rgl_server_*): submit query files as they arrive, wait
    for their count / overlap rows (and p-values with a moment store); p50/p99/p99.9 latency in
    stats().  free_memory (optional): a Python callable returning the free device bytes the server
    should assume when it forms a batch (admission tests); default: the CUDA runtime's figure."""

    def __init__(self, index, workers=0, max_batch_requests=0, batch_intervals=0, hbm_reserve_bytes=0,
                 max_pending_intervals=0, counts_only=False, chunk=0, ctas_per_sm=0, pair_ratio=0,
                 initial_intervals=0, free_memory=None, moments=None, shard_chrom=None, bin_size=0):
        self.index = index
        self._fm = _lib.FREE_MEMORY_FN(lambda user: int(free_memory())) if free_memory else _lib.FREE_MEMORY_FN()
        self._sc = None if shard_chrom is None else np.ascontiguousarray(shard_chrom, np.uint32)
        self.with_stats = moments is not None
        o = _lib.ServerOpts(workers, max_batch_requests, batch_intervals, hbm_reserve_bytes, max_pending_intervals,
                            Context._opts(chunk, ctas_per_sm, counts_only, pair_ratio), initial_intervals, self._fm,
                            None, moments._h if moments is not None else None, _ptr(self._sc),
                            0 if self._sc is None else len(self._sc), bin_size)
        h = C.c_void_p()
        check(load().rgl_server_create(index._h, C.byref(o), C.byref(h)))
        self._h = h
        self._live = {}  # ticket -> arrays that must outlive the request

    def submit(self, blocks, intervals_ptr=None, with_overlap=True):
        """blocks: {shard id: uint32[n,3]} (copied into one array), or, with intervals_ptr (an int
        pointer to page-locked intervals), a list of (shard id, begin, end) element ranges of it.
        Returns the ticket."""
        D = self.index.num_sources
        keep = []
        if intervals_ptr is None:
            items = [(int(k), np.ascontiguousarray(v, np.uint32).reshape(-1, 3)) for k, v in blocks.items()]
            items = [(k, v) for k, v in items if len(v)]
            iv = np.concatenate([v for _, v in items]) if items else np.zeros((0, 3), np.uint32)
            shards = np.array([k for k, _ in items], np.uint32)
            offs = np.zeros(len(items) + 1, np.uint64)
            offs[1:] = np.cumsum([len(v) for _, v in items])
            keep.append(iv)
            ptr = iv.ctypes.data if len(iv) else None
        else:
            shards = np.array([b[0] for b in blocks], np.uint32)
            offs = np.array([blocks[0][1]] + [b[2] for b in blocks], np.uint64) if blocks else np.zeros(1, np.uint64)
            ptr = intervals_ptr
        counts = np.zeros(D, np.uint32)
        bp = np.zeros(D, np.uint64) if with_overlap else None
        pv = None
        if self.with_stats:
            pv = {"p": np.ones(D), "llr": np.zeros(D), "lp": np.zeros(D), "flags": np.zeros(D, np.uint8)}
        keep += [shards, offs, counts, bp, pv]
        req = _lib.Request(len(shards), _ptr(shards), _ptr(offs), C.c_void_p(ptr) if ptr else None, _ptr(counts),
                           _ptr(bp), *((_ptr(pv["p"]), _ptr(pv["llr"]), _ptr(pv["lp"]), _ptr(pv["flags"]))
                                       if pv else (None,) * 4))
        t = C.c_uint64()
        check(load().rgl_server_submit(self._h, C.byref(req), C.byref(t)))
        self._live[t.value] = (keep, counts, bp, pv)
        return t.value

    def wait(self, ticket, timeout_ms=60_000):
        """Returns (counts uint32[D], overlap_bp uint64[D] or None, info dict); with a moment store
        info["pvalues"] holds the request's p, llr, lp (ln p) and flags arrays."""
        info = _lib.RequestInfo()
        check(load().rgl_server_wait(self._h, ticket, timeout_ms, C.byref(info)))
        _, counts, bp, pv = self._live.pop(ticket)
        if info.status:
            raise _lib.RiggleError(info.status, "request failed")
        d = info.as_dict()
        if pv is not None:
            d["pvalues"] = pv
        return counts, bp, d

    def stats(self):
        st = _lib.ServerStats()
        check(load().rgl_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        check(load().rgl_server_reset_stats(self._h))

    def close(self):
        if self._h:
            load().rgl_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceBatch:
    """A file-major query batch whose intervals are in device memory (rgl_batch): block b holds
    intervals [offsets[b], offsets[b+1]) on shard shards[b]; rows[b] (optional) is their file."""

    def __init__(self, num_rows, shards, offsets, d_intervals, rows=None):
        self.num_rows = int(num_rows)
        self.shards = np.ascontiguousarray(shards, np.uint32)
        self.offsets = np.ascontiguousarray(offsets, np.uint64)
        self.rows = None if rows is None else np.ascontiguousarray(rows, np.uint32)
        self.d_intervals = int(d_intervals)
        self.c = _lib.BatchDesc(self.num_rows, len(self.shards), _ptr(self.shards), _ptr(self.rows),
                                _ptr(self.offsets), C.c_void_p(self.d_intervals))

    @property
    def num_intervals(self):
        return int(self.offsets[-1]) if len(self.offsets) else 0


def synth_batch_layout(spec):
    """(offsets uint64[F*C+1], shards uint32[F*C], rows uint32[F*C]) of a file-major batch."""
    nb = spec.num_files * spec.num_chroms
    off = np.empty(nb + 1, np.uint64)
    sh = np.empty(nb, np.uint32)
    rw = np.empty(nb, np.uint32)
    check(load().rgl_synth_batch_layout(C.byref(spec.c), _ptr(off), _ptr(sh), _ptr(rw)))
    return off, sh, rw


def synth_batch_device(spec, offsets, d_out, device=0, stream=None):
    """Generates the batch of `spec` into device memory at d_out (int pointer)."""
    offsets = np.ascontiguousarray(offsets, np.uint64)
    check(load().rgl_synth_batch_device(C.byref(spec.c), device, _ptr(offsets), C.c_void_p(d_out),
                                        C.c_void_p(stream) if stream else None))


class SynthSpec:
    """Seeded synthetic dataset description (rgl_synth_spec)."""

    def __init__(self, seed, chrom_len, file_sizes, broad_fraction=0.0, hotspot_fraction=0.0, num_hotspots=0,
                 sid_base=0):
        self.chrom_len = np.ascontiguousarray(chrom_len, dtype=np.uint32)
        self.file_sizes = np.ascontiguousarray(file_sizes, dtype=np.uint64)
        self.c = _lib.SynthSpec(int(seed), len(self.chrom_len),
                                self.chrom_len.ctypes.data_as(C.POINTER(C.c_uint32)), len(self.file_sizes),
                                self.file_sizes.ctypes.data_as(C.POINTER(C.c_uint64)), float(broad_fraction),
                                float(hotspot_fraction), int(num_hotspots), int(sid_base))

    @property
    def num_files(self):
        return len(self.file_sizes)

    @property
    def num_chroms(self):
        return len(self.chrom_len)

    def chrom_counts(self, file):
        out = np.empty(self.num_chroms, np.uint64)
        check(load().rgl_synth_file_chrom_counts(C.byref(self.c), file, _ptr(out)))
        return out

    def block(self, file, chrom):
        """Intervals of (file, chrom) sorted by (start, end) as uint32[n,3] (start, end, sid)."""
        n = C.c_uint64()
        check(load().rgl_synth_block_host(C.byref(self.c), file, chrom, None, 0, C.byref(n)))
        out = np.empty((n.value, 3), np.uint32)
        check(load().rgl_synth_block_host(C.byref(self.c), file, chrom, _ptr(out), n.value, C.byref(n)))
        return out

    def chrom_layers(self, chrom, min_size=128, growth_factor=4):
        """Host-generated layers of one chromosome: {(chrom, K): (pos uint32[n,2], sid uint32[n])}."""
        tot = C.c_uint64()
        cnt = np.zeros(64, np.uint64)
        check(load().rgl_synth_chrom_layers_host(C.byref(self.c), chrom, min_size, growth_factor, _ptr(cnt), 64,
                                                 None, None, 0, C.byref(tot)))
        pos = np.empty((tot.value, 2), np.uint32)
        sid = np.empty(tot.value, np.uint32)
        check(load().rgl_synth_chrom_layers_host(C.byref(self.c), chrom, min_size, growth_factor, _ptr(cnt), 64,
                                                 _ptr(pos), _ptr(sid), tot.value, C.byref(tot)))
        out, acc = {}, 0
        for k in range(64):
            n = int(cnt[k])
            if n:
                out[(chrom, k)] = (pos[acc:acc + n], sid[acc:acc + n])
                acc += n
        return out

    def file(self, file):
        """All intervals of a file: {chrom index: uint32[n,3]}."""
        return {c: self.block(file, c) for c in range(self.num_chroms)}


CHROM_NAMES_24 = [f"chr{i}" for i in range(1, 23)] + ["chrX", "chrY"]


def synth_chrom_lengths(seed=1, num_chroms=24):
    out = np.empty(num_chroms, np.uint32)
    check(load().rgl_synth_chrom_lengths(seed, num_chroms, _ptr(out)))
    return out


def synth_zipf_sizes(num_files, s=1.1, lo=1000, hi=10_000_000, target=2_000_000_000):
    out = np.empty(num_files, np.uint64)
    check(load().rgl_synth_zipf_sizes(num_files, s, lo, hi, target, _ptr(out)))
    return out


def synth_loguniform_sizes(seed, num_files, lo, hi):
    out = np.empty(num_files, np.uint64)
    check(load().rgl_synth_loguniform_sizes(seed, num_files, lo, hi, _ptr(out)))
    return out


def bucket_layers(blocks, config=None):
    """Host bucketing of interval blocks into the reference's (shard, layer) layers, sorted by start
    (src/tasks/build.rs:190-211).  blocks: iterable of (shard_id, uint32[n,3]).  Returns
    {(shard, layer): (pos uint32[n,2], sid uint32[n])}.  Ties in start keep input order."""
    config = config or LayerConfig()
    per = {}
    for sh, ivs in blocks:
        ivs = np.asarray(ivs, np.uint32).reshape(-1, 3)
        if not len(ivs):
            continue
        sizes = ivs[:, 1] - ivs[:, 0]
        ks = np.array([config.layer_for_size(int(x)) for x in np.unique(sizes)], np.uint32)
        lut = dict(zip(np.unique(sizes).tolist(), ks.tolist()))
        kk = np.vectorize(lut.__getitem__, otypes=[np.uint32])(sizes)
        for k in np.unique(kk):
            per.setdefault((int(sh), int(k)), []).append(ivs[kk == k])
    out = {}
    for key, parts in per.items():
        a = np.concatenate(parts)
        o = np.argsort(a[:, 0], kind="stable")
        a = a[o]
        out[key] = (np.ascontiguousarray(a[:, :2]), np.ascontiguousarray(a[:, 2]))
    return out


# ---------------------------------------------------------------------------------------------
# sliding-window moments and analytic p-values
# ---------------------------------------------------------------------------------------------
HG38_CHROM_SIZES = [  # src/fourier/genome.rs:7-34
    ("chr1", 248_956_422), ("chr2", 242_193_529), ("chr3", 198_295_559), ("chr4", 190_214_555),
    ("chr5", 181_538_259), ("chr6", 170_805_979), ("chr7", 159_345_973), ("chr8", 145_138_636),
    ("chr9", 138_394_717), ("chr10", 133_797_422), ("chr11", 135_086_622), ("chr12", 133_275_309),
    ("chr13", 114_364_328), ("chr14", 107_043_718), ("chr15", 101_991_189), ("chr16", 90_338_345),
    ("chr17", 83_257_441), ("chr18", 80_373_285), ("chr19", 58_617_616), ("chr20", 64_444_167),
    ("chr21", 46_709_983), ("chr22", 50_818_468), ("chrX", 156_040_895), ("chrY", 57_227_415),
]
BIN_SIZE = 100  # src/fourier/genome.rs:3


def compact_index(l):
    return load().rgl_compact_index(int(l))


def moment_grid(n_bins):
    n = load().rgl_moment_grid(int(n_bins), None, 0)
    out = np.empty(n, np.uint64)
    load().rgl_moment_grid(int(n_bins), _ptr(out), n)
    return out


def depth_signal(intervals, n_bins, bin_size=BIN_SIZE, device=0):
    """The reference's f32 coverage signal of intervals (file order) on one chromosome (GPU)."""
    iv = np.ascontiguousarray(np.asarray(intervals, np.uint32).reshape(-1, 3))
    g = np.empty(int(n_bins), np.float32)
    check(load().rgl_depth_signal(device, _ptr(iv), len(iv), int(n_bins), bin_size, _ptr(g)))
    return g


def query_chrom_groups(intervals, bin_size=BIN_SIZE):
    """build_query_chrom_data for one chromosome: (l_int, sum_scale, sum_scale2, count)."""
    iv = np.ascontiguousarray(np.asarray(intervals, np.uint32).reshape(-1, 3))
    ng = C.c_uint64()
    check(load().rgl_query_chrom_groups(_ptr(iv), len(iv), bin_size, None, None, None, None, 0, C.byref(ng)))
    n = ng.value
    li, ss, ss2, cnt = (np.empty(n, np.uint64), np.empty(n, np.float64), np.empty(n, np.float64),
                        np.empty(n, np.uint64))
    check(load().rgl_query_chrom_groups(_ptr(iv), len(iv), bin_size, _ptr(li), _ptr(ss), _ptr(ss2), _ptr(cnt), n,
                                        C.byref(ng)))
    return li, ss, ss2, cnt


class Moments:
    """Device moment store: (mean, var) f32 tables per (source, chromosome)."""

    def __init__(self, num_sources, n_bins, device=0):
        self.n_bins = np.ascontiguousarray(n_bins, np.uint64)
        self.num_sources = num_sources
        h = C.c_void_p()
        check(load().rgl_moments_create(device, num_sources, len(self.n_bins), _ptr(self.n_bins), C.byref(h)))
        self._h = h

    def slots(self, chrom):
        return load().rgl_moments_slots(self._h, chrom)

    def set(self, sid, chrom, mean_var):
        mv = np.ascontiguousarray(np.asarray(mean_var, np.float32).reshape(-1, 2))
        check(load().rgl_moments_set(self._h, sid, chrom, _ptr(mv), len(mv)))

    def build(self, sid, chrom, intervals, bin_size=BIN_SIZE, report=False, precision="fp64"):
        """Moments of one source's intervals (file order) on one chromosome, computed on the GPU;
        precision "fp64" (FP64 FFT) or "fp32c" (compensated FP32, FP64 only in the final reduction)."""
        iv = np.ascontiguousarray(np.asarray(intervals, np.uint32).reshape(-1, 3))
        n = self.slots(chrom)
        mean = np.empty(n, np.float64) if report else None
        var = np.empty(n, np.float64) if report else None
        mode = {"fp64": 0, "fp32c": 1}[precision]
        check(load().rgl_moments_build_ex(self._h, sid, chrom, _ptr(iv), len(iv), bin_size, mode, _ptr(mean),
                                          _ptr(var)))
        return (mean, var) if report else None

    def get(self, sid, chrom):
        n = C.c_uint64()
        check(load().rgl_moments_get(self._h, sid, chrom, None, 0, C.byref(n)))
        out = np.empty((n.value, 2), np.float32)
        check(load().rgl_moments_get(self._h, sid, chrom, _ptr(out), n.value, C.byref(n)))
        return out

    def pvalues(self, row_groups, counts, overlap_bp, bin_size=BIN_SIZE):
        """row_groups: per query row a list of (chrom, (l_int, ss, ss2, count)).

        Returns dense (p, llr, log_p, flags) arrays of shape counts.shape."""
        rows = len(row_groups)
        offs = np.zeros(rows + 1, np.uint64)
        parts = []
        for q, chroms in enumerate(row_groups):
            n = 0
            for c, g in chroms:
                parts.append((c, g))
                n += len(g[0])
            offs[q + 1] = offs[q] + n
        cat = lambda j, dt: np.ascontiguousarray(np.concatenate([g[j] for _, g in parts]) if parts else
                                                 np.zeros(0), dt)
        chrom = np.ascontiguousarray(np.concatenate([np.full(len(g[0]), c, np.uint32) for c, g in parts])
                                     if parts else np.zeros(0, np.uint32))
        li, ss, ss2, cnt = cat(0, np.uint64), cat(1, np.float64), cat(2, np.float64), cat(3, np.uint64)
        b = _lib.PValueBatch(rows, _ptr(offs), _ptr(chrom), _ptr(li), _ptr(ss), _ptr(ss2), _ptr(cnt))
        counts = np.ascontiguousarray(counts, np.uint32)
        overlap_bp = np.ascontiguousarray(overlap_bp, np.uint64)
        p = np.empty(counts.shape, np.float64)
        llr = np.empty(counts.shape, np.float64)
        lp = np.empty(counts.shape, np.float64)
        fl = np.empty(counts.shape, np.uint8)
        check(load().rgl_query_pvalues(self._h, C.byref(b), bin_size, _ptr(counts), _ptr(overlap_bp), _ptr(p),
                                       _ptr(llr), _ptr(lp), _ptr(fl)))
        return p, llr, lp, fl

    def batch_pvalues_device(self, ctx, batch, shard_chrom, d_counts, d_bp, d_p, d_llr, d_log_p, d_flags,
                             bin_size=BIN_SIZE, count_groups=True):
        """Stats stage of a device batch (pointers are device addresses, num_rows x D).  Returns the
        number of query length groups (synchronising), or None with count_groups=False (asynchronous)."""
        sc = np.ascontiguousarray(shard_chrom, np.uint32)
        ng = C.c_uint64()
        check(load().rgl_batch_pvalues_device(ctx._h, self._h, C.byref(batch.c), _ptr(sc), len(sc), bin_size,
                                              C.c_void_p(d_counts), C.c_void_p(d_bp), C.c_void_p(d_p),
                                              C.c_void_p(d_llr), C.c_void_p(d_log_p) if d_log_p else None,
                                              C.c_void_p(d_flags), C.byref(ng) if count_groups else None))
        return ng.value if count_groups else None

    def batch_query_groups(self, ctx, batch, shard_chrom, bin_size=BIN_SIZE):
        """The device-built query length groups of a DeviceBatch (rgl_batch_query_groups): per row a
        list of (chrom, (l_int, sum_scale, sum_scale2, count)), ascending by chromosome."""
        sc = np.ascontiguousarray(shard_chrom, np.uint32)
        rows = batch.num_rows
        offs = np.zeros(rows + 1, np.uint64)
        ng = C.c_uint64()
        args = (ctx._h, self._h, C.byref(batch.c), _ptr(sc), len(sc), bin_size)
        check(load().rgl_batch_query_groups(*args, _ptr(offs), None, None, None, None, None, 0, C.byref(ng)))
        n = ng.value
        ch = np.empty(n, np.uint32)
        li, ss, ss2, cnt = (np.empty(n, np.uint64), np.empty(n, np.float64), np.empty(n, np.float64),
                            np.empty(n, np.uint64))
        check(load().rgl_batch_query_groups(*args, _ptr(offs), _ptr(ch), _ptr(li), _ptr(ss), _ptr(ss2), _ptr(cnt), n,
                                            C.byref(ng)))
        out = []
        for q in range(rows):
            a, b = int(offs[q]), int(offs[q + 1])
            per = []
            for c in np.unique(ch[a:b]):
                k = np.nonzero(ch[a:b] == c)[0] + a
                per.append((int(c), (li[k], ss[k], ss2[k], cnt[k])))
            out.append(per)
        return out

    def close(self):
        if self._h:
            load().rgl_moments_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _names(names):
    if names is None:
        return None, None
    arr = (C.c_char_p * len(names))(*[str(n).encode() for n in names])
    return arr, C.cast(arr, C.c_void_p)


def stats_json(indptr, indices, counts, query_names, db_names, num_sources, observed_bins=None, p_value=None,
               llr=None, flags=None):
    """The reference's StatsOutput JSON (rgl_format_stats_json) of a CSR count matrix, optionally with the
    dense p-value arrays of rgl_query_pvalues (stats mode).  Returns the JSON text."""
    indptr = np.ascontiguousarray(indptr, np.uint64)
    indices = np.ascontiguousarray(indices, np.uint32)
    counts = np.ascontiguousarray(counts, np.uint32)
    rows = len(indptr) - 1
    qa, qp = _names(query_names)
    da, dp = _names(db_names)
    dense = [None if a is None else np.ascontiguousarray(a, dt)
             for a, dt in ((observed_bins, np.float64), (p_value, np.float64), (llr, np.float64), (flags, np.uint8))]
    args = [rows, num_sources, qp, dp, _ptr(indptr), _ptr(indices), _ptr(counts)] + [_ptr(a) for a in dense]
    n = C.c_uint64()
    check(load().rgl_format_stats_json(*args, None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(load().rgl_format_stats_json(*args, buf, n.value, C.byref(n)))
    return buf.raw[:n.value].decode()


def intervals_json(pairs, query_names, db_names, shard_names):
    """The reference's IntervalsOutput JSON (rgl_format_intervals_json) of a uint32[n, 8] pair array in
    rgl_pair layout."""
    pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 8)
    qa, qp = _names(query_names)
    da, dp = _names(db_names)
    sa, sp = _names(shard_names)
    args = [_ptr(pairs), len(pairs), len(query_names), len(db_names), len(shard_names), qp, dp, sp]
    n = C.c_uint64()
    check(load().rgl_format_intervals_json(*args, None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(load().rgl_format_intervals_json(*args, buf, n.value, C.byref(n)))
    return buf.raw[:n.value].decode()


def dense_to_csr_device(ctx, d_counts, num_rows, num_sources, d_bp=None):
    """K9 on the device (rgl_dense_to_csr_device) for device pointers; returns host numpy arrays
    (indptr uint64[rows+1], indices uint32[nnz], values uint32[nnz], bp uint64[nnz] or None)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    indptr = torch.empty(num_rows + 1, dtype=torch.int64, device=dev)
    nnz = C.c_uint64()
    check(load().rgl_dense_to_csr_device(ctx._h, num_rows, num_sources, C.c_void_p(d_counts),
                                         C.c_void_p(d_bp) if d_bp else None, C.c_void_p(indptr.data_ptr()), None,
                                         None, None, 0, C.byref(nnz)))
    n = max(nnz.value, 1)
    ind = torch.empty(n, dtype=torch.int32, device=dev)
    val = torch.empty(n, dtype=torch.int32, device=dev)
    bpv = torch.empty(n, dtype=torch.int64, device=dev) if d_bp else None
    check(load().rgl_dense_to_csr_device(ctx._h, num_rows, num_sources, C.c_void_p(d_counts),
                                         C.c_void_p(d_bp) if d_bp else None, C.c_void_p(indptr.data_ptr()),
                                         C.c_void_p(ind.data_ptr()), C.c_void_p(val.data_ptr()),
                                         C.c_void_p(bpv.data_ptr()) if d_bp else None, nnz.value, C.byref(nnz)))
    k = nnz.value
    return (indptr.cpu().numpy().view(np.uint64), ind[:k].cpu().numpy().view(np.uint32),
            val[:k].cpu().numpy().view(np.uint32), None if bpv is None else bpv[:k].cpu().numpy().view(np.uint64))
