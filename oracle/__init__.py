"""ctypes binding of the CPU oracle (oracle/oracle.cpp) — test infrastructure only.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the product.
Builds oracle/_build/liboracle.so with make when it is missing.  Every function here forwards to a
restatement of the reference's Rust code; see the header of oracle/oracle.cpp.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_P = C.c_void_p


class OrcLayer(C.Structure):
    _fields_ = [("shard", C.c_uint32), ("layer", C.c_uint32), ("count", C.c_uint64), ("pos", _P), ("sid", _P),
                ("jump", _P), ("jump_len", C.c_uint64)]


class OrcQShard(C.Structure):
    _fields_ = [("shard", C.c_uint32), ("count", C.c_uint64), ("ivs", _P)]


_SIGS = {
    "orc_layer_for_size": (C.c_uint32, [C.c_uint32] * 3),
    "orc_layer_max_size": (C.c_uint32, [C.c_uint32] * 3),
    "orc_tile_size": (C.c_uint32, [C.c_uint32] * 3),
    "orc_build_jump_table": (C.c_uint64, [_P, C.c_uint64, C.c_uint32, _P, C.c_uint64]),
    "orc_extend_jump_table": (C.c_uint64, [_P, C.c_uint64, _P, C.c_uint64, C.c_uint32, _P, C.c_uint64]),
    "orc_jump_lookup": (C.c_uint64, [_P, C.c_uint64, C.c_uint32, C.c_uint32]),
    "orc_extend_layer": (None, [_P, _P, C.c_uint64, _P, C.c_uint64, _P, _P]),
    "orc_query_sweep_windowed": (None, [_P, _P, C.c_uint64, C.c_uint32, _P, C.c_uint64, C.c_uint32, _P, C.c_uint64,
                                        C.c_uint32, C.c_uint32, C.c_uint32, _P, _P]),
    "orc_query_database": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P,
                                     C.c_uint32, C.c_int, C.c_int, _P, _P, _P, _P]),
    "orc_query_pairs": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P, _P, C.c_uint64]),
    "orc_bruteforce_counts": (None, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32,
                                     _P, _P]),
    "orc_simd_cumsum_f32": (None, [_P, C.c_uint64]),
    "orc_build_depth_signal": (None, [_P, _P, C.c_uint64, C.c_uint64, C.c_uint32, _P]),
    "orc_compact_index": (C.c_uint64, [C.c_uint64]),
    "orc_moment_grid": (C.c_uint64, [C.c_uint64, _P, C.c_uint64]),
    "orc_autocorr_fft": (None, [_P, C.c_uint64, _P]),
    "orc_prefix_sum_f32_to_f64": (None, [_P, C.c_uint64, _P]),
    "orc_d2_prefix_sum": (None, [_P, C.c_uint64, _P]),
    "orc_window_moments_from_dstar": (None, [_P, C.c_uint64, C.c_uint64, C.POINTER(C.c_double),
                                             C.POINTER(C.c_double)]),
    "orc_moments_from_signal": (C.c_uint64, [_P, C.c_uint64, _P, _P, _P]),
    "orc_moments_exact": (None, [_P, C.c_uint64, _P, C.c_uint64, _P, _P, C.c_int]),
    "orc_erfc": (C.c_double, [C.c_double]),
    "orc_nb_llr": (C.c_int, [C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "orc_poisson_llr": (C.c_int, [C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "orc_query_groups": (C.c_uint64, [_P, _P, C.c_uint64, C.c_uint32, _P, _P, _P, _P]),
    "orc_analytic_stats": (C.c_int, [C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_double,
                                     C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "orc_log_p": (C.c_double, [C.c_double, C.c_int, C.c_double, C.c_double]),
    "orc_synth_chrom_lengths": (None, [C.c_uint64, C.c_uint32, _P]),
    "orc_synth_zipf_sizes": (None, [C.c_uint32, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, _P]),
    "orc_synth_loguniform_sizes": (None, [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, _P]),
    "orc_synth_block": (C.c_uint64, [C.c_uint64, _P, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                     C.c_uint32, C.c_uint32, _P]),
    "orc_synth_chrom_layers": (C.c_uint64, [C.c_uint64, _P, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_double,
                                            C.c_uint32, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P, _P]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(ORACLE_DIR, f) for f in ("oracle.cpp", "synth.cpp")]
        if not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(ORACLE_LIB) < os.path.getmtime(f) for f in srcs):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        L = C.CDLL(ORACLE_LIB)
        for k, (r, a) in _SIGS.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else None


def build_jump_table(starts, tile):
    starts = np.ascontiguousarray(starts, np.uint32)
    n = lib().orc_build_jump_table(_p(starts), len(starts), tile, None, 0)
    out = np.empty(n, np.uint64)
    lib().orc_build_jump_table(_p(starts), len(starts), tile, _p(out), n)
    return out


def extend_jump_table(old, new_starts, tile):
    old = np.ascontiguousarray(old, np.uint64)
    new_starts = np.ascontiguousarray(new_starts, np.uint32)
    n = lib().orc_extend_jump_table(_p(old), len(old), _p(new_starts), len(new_starts), tile, None, 0)
    out = np.empty(n, np.uint64)
    lib().orc_extend_jump_table(_p(old), len(old), _p(new_starts), len(new_starts), tile, _p(out), n)
    return out


def jump_lookup(table, tile, target):
    table = np.ascontiguousarray(table, np.uint64)
    return lib().orc_jump_lookup(_p(table), len(table), tile, target)


def extend_layer(old_pos, old_sid, new_ivs):
    old_pos = np.ascontiguousarray(old_pos, np.uint32).reshape(-1, 2)
    old_sid = np.ascontiguousarray(old_sid, np.uint32)
    new_ivs = np.ascontiguousarray(new_ivs, np.uint32).reshape(-1, 3)
    tot = len(old_sid) + len(new_ivs)
    pos = np.empty((tot, 2), np.uint32)
    sid = np.empty(tot, np.uint32)
    lib().orc_extend_layer(_p(old_pos), _p(old_sid), len(old_sid), _p(new_ivs), len(new_ivs), _p(pos), _p(sid))
    return pos, sid


def query_sweep(db, layer_max, queries, nrows, ncols, bin_size=100):
    """Reference unit-test helper `sweep` (src/sweep/query.rs:144-157): db/queries are (start,end,sid)."""
    db = np.asarray(db, np.uint32).reshape(-1, 3)
    q = np.ascontiguousarray(np.asarray(queries, np.uint32).reshape(-1, 3))
    tile = max(layer_max // 2, 1)
    jt = build_jump_table(db[:, 0], tile) if len(db) else np.zeros(1, np.uint64)
    pos = np.ascontiguousarray(db[:, :2])
    sid = np.ascontiguousarray(db[:, 2])
    counts = np.zeros((nrows, ncols), np.uint32)
    overlap = np.zeros((nrows, ncols), np.float32)
    lib().orc_query_sweep_windowed(_p(pos), _p(sid), len(db), layer_max, _p(jt), len(jt), tile, _p(q), len(q), 0,
                                   ncols, bin_size, _p(counts), _p(overlap))
    return counts, overlap


def _layer_structs(layers, jumps=None):
    """layers: {(shard, layer): (pos[n,2], sid[n])}; jumps: optional {(shard, layer): u64 table}"""
    keep = []
    arr = (OrcLayer * max(1, len(layers)))()
    for i, ((sh, k), (pos, sid)) in enumerate(sorted(layers.items())):
        pos = np.ascontiguousarray(pos, np.uint32).reshape(-1, 2)
        sid = np.ascontiguousarray(sid, np.uint32)
        keep += [pos, sid]
        jt = None
        if jumps is not None and (sh, k) in jumps:
            jt = np.ascontiguousarray(jumps[(sh, k)], np.uint64)
            keep.append(jt)
        arr[i] = OrcLayer(sh, k, len(sid), _p(pos), _p(sid), _p(jt), len(jt) if jt is not None else 0)
    return arr, keep


def jump_tables(layers, min_size=128, growth_factor=4):
    """The `.idx` table a freshly written layer carries (build_jump_table, tile = max_K / 2)."""
    return {key: build_jump_table(pos[:, 0], lib().orc_tile_size(min_size, growth_factor, key[1]))
            for key, (pos, sid) in layers.items()}


def _qshard_structs(qshards):
    keep = []
    arr = (OrcQShard * max(1, len(qshards)))()
    for i, (sh, ivs) in enumerate(sorted(qshards.items())):
        ivs = np.ascontiguousarray(ivs, np.uint32).reshape(-1, 3)
        keep.append(ivs)
        arr[i] = OrcQShard(sh, len(ivs), _p(ivs))
    return arr, keep


def query_database(layers, qshards, rows, num_sources, min_size=128, growth_factor=4, bin_size=100, threads=1,
                   mode=0, jumps=None):
    """Restated counting path of query_database.  Returns counts, overlap_f32, overlap_bp, stats."""
    la, k1 = _layer_structs(layers, jumps)
    qa, k2 = _qshard_structs(qshards)
    counts = np.zeros((rows, num_sources), np.uint32)
    of32 = np.zeros((rows, num_sources), np.float32)
    bp = np.zeros((rows, num_sources), np.uint64)
    st = np.zeros(4, np.uint64)
    lib().orc_query_database(min_size, growth_factor, num_sources, bin_size, len(layers), la, len(qshards), qa, rows,
                             threads, mode, _p(counts), _p(of32), _p(bp), _p(st))
    stats = dict(candidates=int(st[0]), hits=int(st[1]), db_swept=int(st[2]), query_intervals=int(st[3]))
    return counts, of32, bp, stats


def bruteforce(layers, qshards, rows, num_sources, min_size=128, growth_factor=4):
    la, k1 = _layer_structs(layers)
    qa, k2 = _qshard_structs(qshards)
    counts = np.zeros((rows, num_sources), np.uint32)
    bp = np.zeros((rows, num_sources), np.uint64)
    lib().orc_bruteforce_counts(min_size, growth_factor, num_sources, len(layers), la, len(qshards), qa, rows,
                                _p(counts), _p(bp))
    return counts, bp


def query_pairs(layers, qshards, min_size=128, growth_factor=4):
    """Restated `--intervals` mode: every overlapping pair as uint32[n, 8] records (q.start, q.end,
    d.start, d.end, q.sid, d.sid, shard, intersection bp) in the reference's emission order
    (shard, layer, query start, DB start)."""
    la, k1 = _layer_structs(layers)
    qa, k2 = _qshard_structs(qshards)
    n = lib().orc_query_pairs(min_size, growth_factor, len(layers), la, len(qshards), qa, None, 0)
    out = np.empty((n, 8), np.uint32)
    if n:
        lib().orc_query_pairs(min_size, growth_factor, len(layers), la, len(qshards), qa, _p(out), n)
    return out


def depth_signal(starts, ends, n_bins, bin_size=100):
    starts = np.ascontiguousarray(starts, np.uint32)
    ends = np.ascontiguousarray(ends, np.uint32)
    g = np.empty(n_bins, np.float32)
    lib().orc_build_depth_signal(_p(starts), _p(ends), len(starts), n_bins, bin_size, _p(g))
    return g


def cumsum_f32(x):
    g = np.ascontiguousarray(x, np.float32).copy()
    lib().orc_simd_cumsum_f32(_p(g), len(g))
    return g


def moment_grid(n_bins):
    n = lib().orc_moment_grid(n_bins, None, 0)
    out = np.empty(n, np.uint64)
    lib().orc_moment_grid(n_bins, _p(out), n)
    return out


def moments_from_signal(g):
    g = np.ascontiguousarray(g, np.float32)
    n = len(moment_grid(len(g)))
    mv = np.empty(2 * n, np.float32)
    m = np.empty(n, np.float64)
    v = np.empty(n, np.float64)
    lib().orc_moments_from_signal(_p(g), len(g), _p(mv), _p(m), _p(v))
    return mv.reshape(-1, 2), m, v


def moments_exact(g, ls, threads=4):
    """Exact window moments of g for the window lengths ls; threads <= 0 uses every host core."""
    if threads <= 0:
        threads = os.cpu_count() or 1
    g = np.ascontiguousarray(g, np.float32)
    ls = np.ascontiguousarray(ls, np.uint64)
    m = np.empty(len(ls), np.float64)
    v = np.empty(len(ls), np.float64)
    lib().orc_moments_exact(_p(g), len(g), _p(ls), len(ls), _p(m), _p(v), threads)
    return m, v


def autocorr(x):
    x = np.ascontiguousarray(x, np.float64)
    r = np.empty(len(x), np.float64)
    lib().orc_autocorr_fft(_p(x), len(x), _p(r))
    return r


def window_moments_from_g(g, l):
    """Test hook for src/fourier/moments.rs:511-562: d* by plain f64 prefix of g."""
    g = np.asarray(g, np.float32)
    ds = np.zeros(len(g) + 1, np.float64)
    for j in range(1, len(g) + 1):
        ds[j] = ds[j - 1] + float(g[j - 1])
    m, v = C.c_double(), C.c_double()
    lib().orc_window_moments_from_dstar(_p(ds), len(g), l, C.byref(m), C.byref(v))
    return m.value, v.value


def d2_prefix_sum(x):
    x = np.ascontiguousarray(x, np.float64)
    out = np.empty(len(x) + 1, np.float64)
    lib().orc_d2_prefix_sum(_p(x), len(x), _p(out))
    return out


def nb_llr(mu, var, obs):
    out = C.c_double()
    ok = lib().orc_nb_llr(mu, var, obs, C.byref(out))
    return out.value if ok else None


def poisson_llr(mu, obs):
    out = C.c_double()
    ok = lib().orc_poisson_llr(mu, obs, C.byref(out))
    return out.value if ok else None


def erfc(x):
    return lib().orc_erfc(x)


def compact_index(l):
    return lib().orc_compact_index(l)


def query_groups(starts, ends, bin_size=100):
    starts = np.ascontiguousarray(starts, np.uint32)
    ends = np.ascontiguousarray(ends, np.uint32)
    n = len(starts)
    li = np.empty(max(n, 1), np.uint64)
    ss = np.empty(max(n, 1), np.float64)
    ss2 = np.empty(max(n, 1), np.float64)
    cnt = np.empty(max(n, 1), np.uint64)
    g = lib().orc_query_groups(_p(starts), _p(ends), n, bin_size, _p(li), _p(ss), _p(ss2), _p(cnt))
    return li[:g], ss[:g], ss2[:g], cnt[:g]


def analytic_stats(q_chroms, db, observed):
    """q_chroms: list of (chrom_id, (l_int, ss, ss2, count)); db: {chrom_id: (n_bins, mv float32[n,2])}.

    Returns None (no shared chromosome) or (p, llr or None)."""
    nq = len(q_chroms)
    qc = np.array([c for c, _ in q_chroms], np.uint32)
    goff = np.zeros(nq + 1, np.uint64)
    parts = [g for _, g in q_chroms]
    for i, g in enumerate(parts):
        goff[i + 1] = goff[i] + len(g[0])
    cat = lambda j, dt: np.ascontiguousarray(np.concatenate([g[j] for g in parts]) if parts else np.zeros(0), dt)
    gl, gs, gs2, gc = cat(0, np.uint64), cat(1, np.float64), cat(2, np.float64), cat(3, np.uint64)
    ncid = max([c for c, _ in q_chroms] + list(db.keys()) + [0]) + 1
    nb = np.zeros(ncid, np.uint64)
    off = np.zeros(ncid, np.uint64)
    ln = np.zeros(ncid, np.uint64)
    mvs = []
    acc = 0
    for c, (n_bins, mv) in sorted(db.items()):
        mv = np.asarray(mv, np.float32).reshape(-1, 2)
        nb[c] = n_bins
        off[c] = acc
        ln[c] = len(mv)
        acc += len(mv)
        mvs.append(mv)
    mvall = np.ascontiguousarray(np.concatenate(mvs) if mvs else np.zeros((1, 2), np.float32), np.float32)
    p, llr, has = C.c_double(), C.c_double(), C.c_int()
    ok = lib().orc_analytic_stats(nq, _p(qc), _p(goff), _p(gl), _p(gs), _p(gs2), _p(gc), _p(nb), _p(off), _p(ln),
                                  _p(mvall), observed, C.byref(p), C.byref(llr), C.byref(has))
    if not ok:
        return None
    return p.value, (llr.value if has.value else None)


# ---- seeded synthetic workloads (the same bits as the library's generator, without loading it) ----
CHROM_NAMES_24 = [f"chr{i}" for i in range(1, 23)] + ["chrX", "chrY"]


def synth_chrom_lengths(seed=1, num_chroms=24):
    out = np.empty(num_chroms, np.uint32)
    lib().orc_synth_chrom_lengths(seed, num_chroms, _p(out))
    return out


def synth_zipf_sizes(num_files, s=1.1, lo=1000, hi=10_000_000, target=2_000_000_000):
    out = np.empty(num_files, np.uint64)
    lib().orc_synth_zipf_sizes(num_files, s, lo, hi, target, _p(out))
    return out


def synth_loguniform_sizes(seed, num_files, lo, hi):
    out = np.empty(num_files, np.uint64)
    lib().orc_synth_loguniform_sizes(seed, num_files, lo, hi, _p(out))
    return out


class SynthWorkload:
    """A seeded dataset description (seed, chromosome lengths, file sizes, broad / hot-spot shares)
    whose blocks and layers are generated on the CPU."""

    def __init__(self, seed, chrom_len, file_sizes, broad_fraction=0.0, hotspot_fraction=0.0, num_hotspots=0,
                 sid_base=0):
        self.seed = int(seed)
        self.chrom_len = np.ascontiguousarray(chrom_len, np.uint32)
        self.file_sizes = np.ascontiguousarray(file_sizes, np.uint64)
        self.broad, self.hot, self.nhot, self.sid_base = float(broad_fraction), float(hotspot_fraction), \
            int(num_hotspots), int(sid_base)

    @property
    def num_files(self):
        return len(self.file_sizes)

    def block(self, file, chrom):
        args = (self.seed, _p(self.chrom_len), len(self.chrom_len), _p(self.file_sizes), file, chrom, self.broad,
                self.hot, self.nhot, self.sid_base)
        n = lib().orc_synth_block(*args, None)
        out = np.empty((n, 3), np.uint32)
        lib().orc_synth_block(*args, _p(out))
        return out

    def chrom_layers(self, chrom, min_size=128, growth_factor=4):
        """{(chrom, K): (pos uint32[n,2], sid uint32[n])} of every file's intervals on one chromosome."""
        cnt = np.zeros(64, np.uint64)
        args = (self.seed, _p(self.chrom_len), len(self.chrom_len), _p(self.file_sizes), self.num_files, chrom,
                self.broad, self.sid_base, min_size, growth_factor, _p(cnt), 64)
        n = lib().orc_synth_chrom_layers(*args, None, None)
        pos = np.empty((n, 2), np.uint32)
        sid = np.empty(n, np.uint32)
        lib().orc_synth_chrom_layers(*args, _p(pos), _p(sid))
        out, acc = {}, 0
        for k in range(64):
            m = int(cnt[k])
            if m:
                out[(chrom, k)] = (pos[acc:acc + m], sid[acc:acc + m])
                acc += m
        return out


# ---- results (test infrastructure) ---------------------------------------------------------------
def dense_to_csr(counts):
    """query_database's non-zero extraction (src/tasks/query/mod.rs:288-298: rows in order, columns
    in order, val > 0) and build_csr_from_sorted_entries (src/tasks/query/sweep.rs:4-23)."""
    counts = np.asarray(counts)
    rows = counts.shape[0]
    indptr = np.zeros(rows + 1, np.uint64)
    indices, data = [], []
    for r in range(rows):
        cols = np.nonzero(counts[r] > 0)[0]
        indices.extend(cols.tolist())
        data.extend(counts[r, cols].tolist())
        indptr[r + 1] = indptr[r] + len(cols)
    return indptr, np.array(indices, np.uint32), np.array(data, np.uint32)


def json_f64(v):
    """An f64 as serde_json writes it (its shortest-round-trip float printer): plain decimal when
    the decimal exponent kk (10^(kk-1) <= |v| < 10^kk) satisfies -5 < kk <= 16, with ".0" on
    integers; else d.ddde<exp>.  Digits from Python's shortest repr."""
    import decimal
    import math

    if not math.isfinite(v):
        return "null"
    if v == 0.0:
        return "-0.0" if math.copysign(1.0, v) < 0 else "0.0"
    t = decimal.Decimal(repr(v)).as_tuple()
    digits = "".join(map(str, t.digits)).rstrip("0") or "0"
    exp = t.exponent + (len(t.digits) - len(digits))  # v = digits x 10^exp
    length = len(digits)
    kk = length + exp
    sign = "-" if t.sign else ""
    if 0 <= exp and kk <= 16:
        return sign + digits + "0" * exp + ".0"
    if 0 < kk <= 16:
        return sign + digits[:kk] + "." + digits[kk:]
    if -5 < kk <= 0:
        return sign + "0." + "0" * (-kk) + digits
    return sign + digits[0] + ("." + digits[1:] if length > 1 else "") + "e" + str(kk - 1)


def json_pretty(results_key, objects):
    """serde_json::to_string_pretty of a struct with one Vec field of flat structs: objects is a list
    of [(key, value)] with value str, int or float (StatsOutput / IntervalsOutput,
    src/stats/mod.rs:1-60)."""
    import json

    if not objects:
        return '{\n  "%s": []\n}' % results_key
    parts = []
    for obj in objects:
        lines = []
        for k, v in obj:
            if isinstance(v, str):
                val = json.dumps(v, ensure_ascii=False)
            elif isinstance(v, float):
                val = json_f64(v)
            else:
                val = str(int(v))
            lines.append('      "%s": %s' % (k, val))
        parts.append("    {\n" + ",\n".join(lines) + "\n    }")
    return '{\n  "%s": [\n' % results_key + ",\n".join(parts) + "\n  ]\n}"
