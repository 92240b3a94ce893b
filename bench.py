#!/usr/bin/env python
"""Benchmark of the interval sweep on B200: intervals swept per second, batched vs plain, and the
serving loop's latency, counts exact.

One JSON line with three parts:
  value (primary, the GPU-scale plain configuration): 24 chromosomes with lengths uniform in
    [50M, 250M] bp, a database of 1,000 files with rank-Zipf(1.1) sizes clamped to [1e3, 1e7]
    intervals summing to 2e9 (log-normal lengths, median 500 bp, sigma 1, clipped to [20, 100k], plus
    5% log-uniform [10k, 1M] broad intervals), u32 start/end/file-id resident in HBM (~24 GB), and one
    query file of 1e5 intervals per step (a different seeded file every step).  A step is one pass of
    the hot path: sort the query file, partition the candidate ranges, sweep and tally the 1 x 1000
    count vector and overlap base pairs.  Carries roofline, cpu_baseline, e2e and clocks.
  "batched" / "batched_2e9": 4,096 query files (log-uniform [1e2, 1e6] intervals, 10% in 1 Mbp hot
    spots, sorted by start within each chromosome) against the 64-file x 50k database and against
    the 2e9-interval database, in one call (CUDA graph replay; autotuned launch shape against the
    small database), next to the plain form on the same files (one call per file), with the results
    compared cell by cell; the same files in generation order beside; the stats stage (FP64 p-value
    of every cell) and the host-input form.
  "serving": Poisson arrivals at 200 query files/s (log-uniform [1e3, 1e6] intervals) against the
    resident 2e9-interval database through the request server, with p-values: p50/p99/p99.9 latency
    and sustained rate, continuous batching vs one query file per launch; "high_load" repeats it at
    twice the rate and "overload" at four times, beyond what one file per launch sustains.
  "precision": FFT sliding-window moments at 2^20..2^26 FFT points in FP64 and compensated FP32,
    errors against the oracle's exact moments.

"intervals swept" = query intervals + database intervals in the union of the reference's candidate
ranges [q.start - layer_max_K, q.end) over all (shard, layer), per query file (computed by the
pipeline itself).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl riggle|reference]
       [--workload plain|config1] [--batch-files F] [--serve-seconds S] [--only all|plain|batched|serving]
For N > 1 launch with torch.distributed.run: every rank holds a replica of the index and sweeps its
own query files (weak scaling, no data-path collective); timing is the max over ranks.  The batched
and serving parts run at N = 1 only.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "intervals swept/s + p99 latency, batched vs plain, 1 B200, counts exact"
UNIT = "intervals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["riggle", "reference"], default="riggle")
    ap.add_argument("--workload", choices=["plain", "config1"], default="plain")
    ap.add_argument("--query-size", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--pair-ratio", type=int, default=0,
                    help="candidate/union ratio below which a range is swept pair by pair (0 = library default)")
    ap.add_argument("--db-intervals", type=int, default=2_000_000_000,
                    help="database size of the plain workload (smaller values for profiling captures)")
    ap.add_argument("--chroms", type=int, default=24,
                    help="keep only the first N chromosomes, scaling database and query sizes by their share "
                         "of the genome (same per-bp density; for profiling captures)")
    ap.add_argument("--batch-files", type=int, default=4096,
                    help="query files of the batched measurement (0 skips it)")
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--batch-db", choices=["both", "config1", "config2"], default="both",
                    help="database(s) of the batched part")
    ap.add_argument("--batch-tune", action="store_true", help="autotune the batched part against config 2 too")
    ap.add_argument("--serve-seconds", type=float, default=5.0,
                    help="length of the Poisson arrival trace of the serving measurement (0 skips it)")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--precision-sizes", type=int, default=4,
                    help="signal sizes of the precision part (2^19, 2^21, 2^23, 2^25 bins; 0 skips it)")
    ap.add_argument("--only", choices=["all", "plain", "batched", "serving", "precision"], default="all",
                    help="run one part only (profiling captures)")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# workload definitions
# ---------------------------------------------------------------------------------------------
def generator(cpu=False):
    """The seeded workload generator: the library's, or (cpu=True) the oracle's restatement of it,
    which gives the same bits without loading the GPU library (the CPU reference arm)."""
    if cpu:
        import oracle as O

        return O, O.SynthWorkload
    import riggle_b200 as rg

    return rg, rg.SynthSpec


def workload_spec(name, db_intervals=2_000_000_000, chroms=24, cpu=False):
    gen, Spec = generator(cpu)
    cl = gen.synth_chrom_lengths(1, 24)
    share = float(cl[:chroms].sum()) / float(cl.sum())
    cl = cl[:chroms]
    if name == "plain":
        sizes = gen.synth_zipf_sizes(1000, 1.1, max(1, int(1000 * share)), max(1, int(10_000_000 * share)),
                                     int(db_intervals * share))
        db = Spec(2, cl, sizes, broad_fraction=0.05)
        qsize = int(round(100_000 * share))
        desc = {"workload": f"plain GPU-scale sweep: 1,000-file Zipf(1.1) database, {db_intervals:.3g} intervals "
                            "(5% broad 10k-1M bp), one 1e5-interval query file per launch",
                "db_files": 1000, "db_intervals": int(sizes.sum()), "query_intervals_per_step": qsize,
                "chromosomes": len(cl), "bin_size": 100, "layer_config": "min_size 128, growth_factor 4"}
    else:
        sizes = np.full(64, int(round(50_000 * share)), np.uint64)
        db = Spec(2, cl, sizes)
        qsize = int(round(10_000 * share))
        desc = {"workload": "plain CPU-runnable sweep: 64-file database x 50k intervals, one 1e4-interval "
                            "query file per launch",
                "db_files": 64, "db_intervals": int(sizes.sum()), "query_intervals_per_step": qsize,
                "chromosomes": len(cl), "bin_size": 100, "layer_config": "min_size 128, growth_factor 4"}
    desc["reference_arm_sample"] = ("the shortest chromosome of each step's query file against all database files "
                                    "(the CPU reference arm and cpu_baseline time this bounded sample)")
    return cl, db, qsize, desc


def query_file(cl, seed, qsize, cpu=False):
    """One seeded query file as AoS (start, end, row=0) grouped by chromosome + shard offsets."""
    _, Spec = generator(cpu)
    q = Spec(seed, cl, [qsize])
    blocks = [q.block(0, c) for c in range(len(cl))]
    offs = np.zeros(len(cl) + 1, np.uint64)
    for c, b in enumerate(blocks):
        offs[c + 1] = offs[c] + len(b)
    ivs = np.concatenate(blocks).astype(np.uint32)
    ivs[:, 2] = 0
    return np.ascontiguousarray(ivs), offs, blocks


# ---------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples every 50 ms, each stamped on arrival; stop(t0, t1) keeps the samples taken
    inside the timed region [t0, t1] (perf_counter), or, for a region shorter than the sampling
    period, the samples within 250 ms of it (marked in "window")."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self, t0=None, t1=None):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        lines = self.lines
        window = "timed region"
        if t0 is not None:
            inside = [x for x in lines if t0 <= x[0] <= t1]
            if not inside:
                inside = [x for x in lines if t0 - 0.25 <= x[0] <= t1 + 0.25]
                window = "timed region +- 250 ms (region shorter than the 50 ms sampling period allows)"
            lines = inside
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, ln in lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "window": window}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------------
# CPU side: the oracle's restatement of the reference's query path on a bounded sample
# ---------------------------------------------------------------------------------------------
def sample_layers(db, chroms):
    """Host-generated layers (and their jump tables) of the sampled chromosomes."""
    import oracle as O

    out = {}
    for c in chroms:
        layers = db.chrom_layers(c)
        out[c] = (layers, O.jump_tables(layers))
    return out


def cpu_sample(db, layers_by_chrom, qblocks, threads, mode):
    import oracle as O

    swept = nq = 0
    t = 0.0
    for c, (layers, jumps) in layers_by_chrom.items():
        q = qblocks[c]
        t0 = time.perf_counter()
        _, _, _, st = O.query_database(layers, {c: q}, 1, db.num_files, threads=threads, mode=mode, jumps=jumps)
        t += time.perf_counter() - t0
        swept += st["db_swept"]
        nq += st["query_intervals"]
    return swept + nq, t


def pick_sample(cl, workload):
    # the shortest chromosomes keep the CPU sample to tens of seconds
    order = np.argsort(cl)
    return [int(order[0])] if workload == "plain" else [int(x) for x in order[:6]]


# ---------------------------------------------------------------------------------------------
def run_reference(args, rank, world):
    """The reference's CPU algorithm (the oracle's restatement; the Rust crate cannot be built on
    this image) on the host cores, on a bounded sample of the same workload."""
    if rank != 0:
        return
    import oracle as O

    # inputs from the oracle's generator: this arm never loads the GPU library
    cl, db, qsize, desc = workload_spec(args.workload, args.db_intervals, args.chroms, cpu=True)
    qsize = args.query_size or qsize
    cores = os.cpu_count() or 1
    chroms = pick_sample(cl, args.workload)
    sl = sample_layers(db, chroms)
    vals = []
    for step in range(args.warmup + args.steps):
        _, _, blocks = query_file(cl, 1000 + step, qsize, cpu=True)
        n, t = cpu_sample(db, sl, blocks, cores, 1)
        if step >= args.warmup:
            vals.append(n / t)
    v = float(np.mean(vals))
    sample = (f"chromosome(s) {[O.CHROM_NAMES_24[c] for c in chroms]} of each step's query file against all "
              f"database files, query-block parallel restatement of src/sweep/query.rs on {cores} threads")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)", "config": desc,
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_riggle(args, rank, world, local_rank, dist):
    import torch

    import riggle_b200 as rg
    from riggle_b200 import _lib

    lib = rg.load()
    dev = local_rank
    torch.cuda.set_device(dev)
    cl, db, qsize, desc = workload_spec(args.workload, args.db_intervals, args.chroms)
    qsize = args.query_size or qsize
    t0 = time.time()
    idx = rg.Index.synth(db, device=dev)
    build_s = time.time() - t0
    ctx = rg.Context(idx)
    D = idx.num_sources
    nfiles = args.warmup + args.steps
    files = [query_file(cl, 1000 + 7919 * rank + i, qsize) for i in range(nfiles)]
    maxn = max(len(f[0]) for f in files)
    ctx.reserve(maxn, 1)

    stream = torch.cuda.ExternalStream(ctx.stream)
    shard_ids = np.arange(len(cl), dtype=np.uint32)
    opts = _lib.QueryOpts(args.chunk, args.ctas_per_sm, 0, 0, args.pair_ratio)
    d_files = [torch.from_numpy(f[0].view(np.int32)).to(f"cuda:{dev}") for f in files]
    d_counts = torch.zeros((1, D), dtype=torch.int32, device=f"cuda:{dev}")
    d_bp = torch.zeros((1, D), dtype=torch.int64, device=f"cuda:{dev}")
    torch.cuda.synchronize()

    def dev_step(i, stats=None):
        f = files[i]
        _lib.check(lib.rgl_query_counts_device(ctx._h, 1, len(cl), C.c_void_p(shard_ids.ctypes.data),
                                               C.c_void_p(f[1].ctypes.data), C.c_void_p(d_files[i].data_ptr()),
                                               C.byref(opts), C.c_void_p(d_counts.data_ptr()),
                                               C.c_void_p(d_bp.data_ptr()), C.byref(stats) if stats else None))

    # per-file work (intervals swept) from one untimed pass with stats
    swept = []
    for i in range(nfiles):
        st = _lib.QueryStats()
        dev_step(i, st)
        swept.append(st.db_swept + st.query_intervals)
        if i == 0:
            first_stats = st.as_dict()
    work = np.array(swept, np.float64)

    # ---- device-resident timing (value) ----
    clocks = ClockSampler(dev).start()
    time.sleep(0.3)  # the sampler's first line
    for i in range(args.warmup):
        dev_step(i)
    _lib.check(lib.rgl_context_check(ctx._h))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    lib.rgl_context_set_timing(ctx._h, 1)
    tc0 = time.perf_counter()
    torch.cuda.profiler.start()  # the profiled range under `ncu --profile-from-start off`
    e0.record(stream)
    for i in range(args.warmup, nfiles):
        dev_step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    tc1 = time.perf_counter()
    sweep_ms = C.c_float()
    launches = C.c_uint32()
    _lib.check(lib.rgl_context_sweep_times(ctx._h, C.byref(sweep_ms), C.byref(launches)))
    lib.rgl_context_set_timing(ctx._h, 0)
    clk = clocks.stop(tc0, tc1)
    _lib.check(lib.rgl_context_check(ctx._h))
    ms = e0.elapsed_time(e1)
    units = float(work[args.warmup:].sum())
    if dist:
        t = torch.tensor([ms, units], dtype=torch.float64, device=f"cuda:{dev}")
        tmax = t.clone()
        torch.distributed.all_reduce(tmax[:1], op=torch.distributed.ReduceOp.MAX)
        tsum = t.clone()
        torch.distributed.all_reduce(tsum[1:], op=torch.distributed.ReduceOp.SUM)
        ms, units = float(tmax[0]), float(tsum[1])
    value = units / (ms / 1e3)

    # ---- end to end through the host C ABI with pinned buffers (e2e) ----
    pin_q = []
    for f in files:
        p = C.c_void_p()
        _lib.check(lib.rgl_host_alloc(f[0].nbytes, C.byref(p)))
        C.memmove(p, f[0].ctypes.data, f[0].nbytes)
        pin_q.append(p)
    pc, pb = C.c_void_p(), C.c_void_p()
    _lib.check(lib.rgl_host_alloc(D * 4, C.byref(pc)))
    _lib.check(lib.rgl_host_alloc(D * 8, C.byref(pb)))

    def host_step(i):
        f = files[i]
        sh = (_lib.QueryShard * len(cl))()
        for c in range(len(cl)):
            n = int(f[1][c + 1] - f[1][c])
            sh[c] = _lib.QueryShard(None, c, n, C.c_void_p(pin_q[i].value + int(f[1][c]) * 12) if n else None)
        batch = _lib.QueryBatch(1, len(cl), sh)
        _lib.check(lib.rgl_query_counts(ctx._h, C.byref(batch), C.byref(opts), pc, pb, None))

    for i in range(args.warmup):
        host_step(i)
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(args.warmup, nfiles):
        host_step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ems], dtype=torch.float64, device=f"cuda:{dev}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ems = float(t[0])
    e2e = units / (ems / 1e3)
    h2d = float(np.mean([f[0].nbytes for f in files[args.warmup:]]))

    # ---- roofline of the sweep kernel ----
    per_launch_ms = sweep_ms.value / max(1, launches.value)
    # algorithmic bytes: 12 per swept DB interval (pos 8 + sid 4), 12 per query interval, 12 per output cell
    qn = np.array([len(f[0]) for f in files[args.warmup:]], np.float64)
    dbs = work[args.warmup:] - qn
    alg_bytes = float(np.mean(12 * dbs + 12 * qn + 12 * D))
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "traffic_note": "DRAM bytes per launch are measured by ncu, not in this run: the "
                                                  "committed capture of this workload is summarised in profiles/",
                "kernel": "k_sweep + k_pairs (sweep stage)", "peak_source": peak_kind,
                "sweep_ms_per_launch": per_launch_ms, "algorithmic_bytes_per_launch": alg_bytes}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle  # noqa: F401  (builds the oracle if needed)

        chroms = pick_sample(cl, args.workload)
        n, t = cpu_sample(db, sample_layers(db, chroms), files[args.warmup][2], 1, 0)
        cpu = {"value": n / t, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{[rg.CHROM_NAMES_24[c] for c in chroms]} of one query file against all database files; "
                         "restatement of query_database/query_sweep_windowed with the reference's parallel "
                         "structure (one query file = one 64-row window = one thread)"}

    own_launches = first_stats["kernel_launches"]
    out = None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
               "config": dict(desc, l2="database (24 GB) and per-step swept set exceed L2; a different query "
                                        "file each step", parallelism=f"replicas x{world}" if world > 1 else "1 GPU",
                              chunk=first_stats["chunk"], ctas_per_sm=first_stats["ctas_per_sm"]),
               "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": D * 12,
                       "ms_per_step": ems / args.steps},
               "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
               "gpu_launches": own_launches * args.steps,
               "extra": {"index_build_s": build_s, "db_swept_first": first_stats["db_swept"],
                         "ranges_first": first_stats["ranges"], "device_ms_first": first_stats["device_ms"],
                         "sweep_ms_first": first_stats["sweep_ms"], "own_kernels_per_step": own_launches}}
    for p in pin_q:
        lib.rgl_host_free(p)
    lib.rgl_host_free(pc)
    lib.rgl_host_free(pb)
    ctx.close()
    return out, (idx, db)


# ---------------------------------------------------------------------------------------------
# batched form (4,096 query files in one call) against the plain one-file-per-launch form
# ---------------------------------------------------------------------------------------------
def batched_workload(nfiles):
    """The 64-file x 50k database and a seeded batch of query files with log-uniform [1e2, 1e6] sizes,
    10% of each file's intervals in 1 Mbp hot spots (8 spots per chromosome shared by all files)."""
    import riggle_b200 as rg

    cl = rg.synth_chrom_lengths(1, 24)
    db = rg.SynthSpec(2, cl, np.full(64, 50_000, np.uint64))
    sizes = rg.synth_loguniform_sizes(4242, nfiles, 100, 1_000_000) if nfiles else np.zeros(0, np.uint64)
    q = rg.SynthSpec(5000, cl, sizes, hotspot_fraction=0.1, num_hotspots=8)
    return cl, db, q


def sort_blocks_device(t_iv, off, dev):
    """Sorts every block of a device batch (int32 [n, 3] intervals, block offsets off) by (start,
    end) in place, as the host generator returns a (file, chromosome) block and as BED files are
    usually stored: two stable device sorts, by end and then by (block, start)."""
    import torch

    cnt = torch.from_numpy(np.diff(np.asarray(off, np.int64))).to(f"cuda:{dev}")
    blk = torch.repeat_interleave(torch.arange(len(cnt), device=f"cuda:{dev}", dtype=torch.int64), cnt)
    s = t_iv[:, 0].to(torch.int64) & 0xFFFFFFFF
    e = t_iv[:, 1].to(torch.int64) & 0xFFFFFFFF
    o1 = torch.sort(e, stable=True).indices
    del e
    o2 = torch.sort((blk[o1] << 32) | s[o1], stable=True).indices
    del s, blk
    t_iv.copy_(t_iv[o1[o2]])
    del o1, o2
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # the sorts' temporaries back to the device for the library's buffers


def run_batched(args, dev, which, big=None):
    """The batched form (one call over all query files, CUDA-graph replay) against the plain form (one
    call per file) on the same 4,096 files, results compared cell by cell.  which = "config1": the
    64-file x 50k database; "config2": the 2e9-interval database of the plain part (big = (index,
    database spec)).  Units are the per-file candidate unions summed (the plain form's work), counted
    by an untimed region-free batched pass, so both forms are measured in the same units."""
    import torch

    import riggle_b200 as rg
    from riggle_b200 import _lib

    lib = rg.load()
    cl, dbspec, qspec = batched_workload(args.batch_files)
    if which == "config1":
        idx = rg.Index.synth(dbspec, device=dev)
        db_desc = "the 64-file x 50k database (config 1)"
    else:
        idx, dbspec = big
        db_desc = (f"the 1,000-file database of {int(np.sum(dbspec.file_sizes)):.3g} intervals (config 2, "
                   "resident 24 GB)")
    D = idx.num_sources
    off, sh, rw = rg.synth_batch_layout(qspec)
    N, F = int(off[-1]), qspec.num_files
    cuda = f"cuda:{dev}"
    t_iv = torch.empty((N, 3), dtype=torch.int32, device=cuda)
    rg.synth_batch_device(qspec, off, t_iv.data_ptr(), device=dev)
    ctx = rg.Context(idx)
    batch = rg.DeviceBatch(F, sh, off, t_iv.data_ptr(), rw)
    dc = torch.empty((F, D), dtype=torch.int32, device=cuda)
    dbp = torch.empty((F, D), dtype=torch.int64, device=cuda)
    # units: the per-file unions (no region split) and the query intervals
    st0 = ctx.query_batch_device(batch, dc.data_ptr(), dbp.data_ptr(), region_bits=_lib.RGL_BATCH_NO_REGIONS)
    units = float(st0["db_swept"] + st0["query_intervals"])
    tune = which == "config1" or args.batch_tune
    best, trials, tune_s = None, [], 0.0
    if tune:
        t0 = time.perf_counter()
        best, trials = ctx.autotune(batch)
        tune_s = time.perf_counter() - t0
    # the files as generated (intervals in random order within each chromosome): the key sorts do
    # the full work; then the same files sorted by start, as BED files are, for everything below
    for _ in range(2):
        ctx.query_batch_device(batch, dc.data_ptr(), dbp.data_ptr(), graph=True, tuned=tune)
    u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ustream = torch.cuda.ExternalStream(ctx.stream)
    torch.cuda.synchronize()
    u0.record(ustream)
    for _ in range(args.batch_steps):
        ctx.query_batch_device(batch, dc.data_ptr(), dbp.data_ptr(), graph=True, tuned=tune, stats=False)
    u1.record(ustream)
    torch.cuda.synchronize()
    ms_unsorted = u0.elapsed_time(u1) / args.batch_steps
    uc, ub = dc.clone(), dbp.clone()
    sort_blocks_device(t_iv, off, dev)
    # capture, then replays: the timed steps launch the cached graph
    for _ in range(2):
        st = ctx.query_batch_device(batch, dc.data_ptr(), dbp.data_ptr(), graph=True, tuned=tune)
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dev).start()
    time.sleep(0.3)  # the sampler's first line
    torch.cuda.synchronize()
    tc0 = time.perf_counter()
    torch.cuda.profiler.start()  # the profiled range under `ncu --profile-from-start off`
    e0.record(stream)
    for _ in range(args.batch_steps):
        ctx.query_batch_device(batch, dc.data_ptr(), dbp.data_ptr(), graph=True, tuned=tune, stats=False)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    clk = clocks.stop(tc0, time.perf_counter())
    ctx.check()
    ms = e0.elapsed_time(e1) / args.batch_steps
    value = units / (ms / 1e3)
    bc = dc.cpu().numpy().view(np.uint32)
    bb = dbp.cpu().numpy().view(np.uint64)
    unsorted_equal = bool(torch.equal(uc, dc) and torch.equal(ub, dbp))
    del uc, ub

    # the stats stage (FP64 p-value matrix of every (file, source) cell) on a moment store of the
    # database: built on the device from the database's own intervals (config 1), or tables of the
    # right shape (config 2, whose 24,000 (source, chromosome) signals are not rebuilt here)
    from riggle_b200 import api

    t0 = time.perf_counter()
    if which == "config1":
        mom = api.Moments(D, (np.asarray(cl, np.uint64) + 99) // 100, device=dev)
        for f in range(dbspec.num_files):
            for c in range(len(cl)):
                blk = dbspec.block(f, c)
                if len(blk):
                    mom.build(f, c, blk)
        mom_kind = "built on the device from the database intervals (FP64 FFT moments)"
    else:
        mom = synthetic_moments(D, cl, dbspec.file_sizes, dev)
        mom_kind = "synthetic tables of the store's shape (the stage's cost does not depend on the values)"
    moments_s = time.perf_counter() - t0
    shard_chrom = np.arange(len(cl), dtype=np.uint32)
    pv = {k: torch.empty((F, D), dtype=dt, device=cuda)
          for k, dt in (("p", torch.float64), ("llr", torch.float64), ("lp", torch.float64), ("f", torch.uint8))}

    def stats_stage(count_groups=False):
        return mom.batch_pvalues_device(ctx, batch, shard_chrom, dc.data_ptr(), dbp.data_ptr(), pv["p"].data_ptr(),
                                        pv["llr"].data_ptr(), pv["lp"].data_ptr(), pv["f"].data_ptr(),
                                        count_groups=count_groups)

    ngroups = stats_stage(True)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()  # a second profiled range: counts plus the stats stage
    e0.record(stream)
    for _ in range(args.batch_steps):
        ctx.query_batch_device(batch, dc.data_ptr(), dbp.data_ptr(), graph=True, tuned=tune, stats=False)
        stats_stage()
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    ctx.check()
    ms_pv = e0.elapsed_time(e1) / args.batch_steps
    emitted = int((pv["f"] & 1).sum().item())
    min_lp = float(pv["lp"].min().item())
    del pv

    # the plain form on the same files: one rgl_query_counts_device call (one pipeline) per file
    t_plain = t_iv.clone()
    t_plain[:, 2] = 0
    pc = torch.empty((F, D), dtype=torch.int32, device=cuda)
    pb = torch.empty((F, D), dtype=torch.int64, device=cuda)
    shard_ids = np.arange(len(cl), dtype=np.uint32)
    opts = _lib.QueryOpts(0, 0, 0, 0, 0)
    C_ = len(cl)
    offs_f = [np.ascontiguousarray(off[f * C_:(f + 1) * C_ + 1]) for f in range(F)]
    ctx.reserve(int(max(qspec.file_sizes)) + 16, 1)

    def plain_pass(files):
        for f in files:
            _lib.check(lib.rgl_query_counts_device(ctx._h, 1, C_, C.c_void_p(shard_ids.ctypes.data),
                                                   C.c_void_p(offs_f[f].ctypes.data), C.c_void_p(t_plain.data_ptr()),
                                                   C.byref(opts), C.c_void_p(pc.data_ptr() + f * D * 4),
                                                   C.c_void_p(pb.data_ptr() + f * D * 8), None))

    plain_pass(range(min(F, 64)))
    torch.cuda.synchronize()
    e0.record(stream)
    plain_pass(range(F))
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.check()
    plain_ms = e0.elapsed_time(e1)
    plain_value = units / (plain_ms / 1e3)
    exact = bool((pc.cpu().numpy().view(np.uint32) == bc).all() and (pb.cpu().numpy().view(np.uint64) == bb).all())
    if not exact:
        raise RuntimeError("batched and plain forms disagree")
    del t_plain, pc, pb

    # end to end: host intervals in page-locked memory, copies overlapped with the sweep
    hp = C.c_void_p()
    _lib.check(lib.rgl_host_alloc(N * 12, C.byref(hp)))
    hv = np.ctypeslib.as_array((C.c_uint32 * (N * 3)).from_address(hp.value))
    hv[:] = t_iv.cpu().numpy().view(np.uint32).reshape(-1)
    hc = np.empty((F, D), np.uint32)
    hb = np.empty((F, D), np.uint64)
    ctx.query_batch_host(batch, hp.value, tuned=tune, out=(hc, hb))
    walls = []
    for _ in range(2):
        t0 = time.perf_counter()
        ctx.query_batch_host(batch, hp.value, tuned=tune, out=(hc, hb))
        walls.append(time.perf_counter() - t0)
    e2e_s = min(walls)
    if not ((hc == bc).all() and (hb == bb).all()):
        raise RuntimeError("host-input batch disagrees")
    lib.rgl_host_free(hp)

    # CPU: the oracle's restatement on a bounded sample of the batch's files
    cpu = None
    if not args.no_cpu_baseline:
        import oracle as O

        host = t_iv.cpu().numpy().view(np.uint32)
        if which == "config1":
            sample, chroms = list(range(0, F, max(1, F // 48)))[:48], list(range(C_))
        else:  # the 2e9 database: the shortest chromosome of a few files
            sample, chroms = list(range(0, F, max(1, F // 6)))[:6], [int(np.argmin(cl))]
        layers = {}
        for c in chroms:
            layers.update(dbspec.chrom_layers(c))
        jumps = O.jump_tables(layers)
        n_s = 0.0
        t_s = 0.0
        for f in sample:
            per = {}
            for c in chroms:
                a = host[int(off[f * C_ + c]):int(off[f * C_ + c + 1])].copy()
                if len(a):
                    a[:, 2] = 0
                    per[c] = a
            t0 = time.perf_counter()
            _, _, _, ost = O.query_database(layers, per, 1, D, threads=1, mode=0, jumps=jumps)
            t_s += time.perf_counter() - t0
            n_s += ost["db_swept"] + ost["query_intervals"]
        cpu = {"value": n_s / max(t_s, 1e-9), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{len(sample)} of the {F} query files, chromosomes "
                         f"{[rg.CHROM_NAMES_24[c] for c in chroms] if len(chroms) < 24 else 'all'}, restatement "
                         "of query_database/query_sweep_windowed, one thread per query file"}
    peak, peak_kind = measured_peak()
    nsub = max(1, int(st["sub_batches"]))
    db_bytes = 12.0 * float(idx.num_intervals)
    alg_units = 12.0 * units + 12.0 * F * D
    out = {"workload": f"batched: {F} query files, log-uniform [1e2, 1e6] intervals (10% in 1 Mbp hot spots), "
                       f"sorted by start within each chromosome as BED files are, against {db_desc}, one call "
                       "(graph replay, "
                       + ("autotuned" if tune else "default") + " launch shape)",
           "value": value, "unit": UNIT, "ms_per_step": ms, "steps": args.batch_steps, "query_files": F,
           "query_intervals": int(st0["query_intervals"]), "db_swept_per_file_unions": int(st0["db_swept"]),
           "db_swept_region_order": int(st["db_swept"]), "sub_batches": st["sub_batches"],
           "graph_nodes": st["graph_nodes"], "gpu_launches_per_step": st["kernel_launches"],
           "tuned": best, "tune_trials": len(trials), "tune_s": tune_s,
           "plain": {"value": plain_value, "ms_per_step": plain_ms,
                     "form": "one rgl_query_counts_device call per query file, same files, same units"},
           "batched_vs_plain": value / plain_value, "counts_exact_vs_plain": exact,
           "unsorted_input": {"ms_per_step": ms_unsorted, "value": units / (ms_unsorted / 1e3),
                              "counts_equal_sorted": unsorted_equal,
                              "note": "the same files with their intervals in generation order: the key sorts "
                                      "sort every block instead of copying it through"},
           "roofline": {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_source": peak_kind,
                        "achieved_unit_bytes": alg_units / (ms / 1e3) / 1e9,
                        "frac_unit_bytes": alg_units / (ms / 1e3) / 1e9 / peak,
                        "unit_bytes_note": "12 B per swept database interval of each file's union, per query interval "
                                           "and per output cell: the plain form reads these from HBM; the batched "
                                           "form reads a region of the database once from HBM for all rows of a "
                                           "sub-batch and from L2 for the others",
                        "achieved_read_once": (db_bytes * nsub + 12.0 * N + 12.0 * F * D) / (ms / 1e3) / 1e9,
                        "read_once_note": "the database read once per sub-batch (12 B x database intervals x "
                                          f"{nsub} sub-batches) plus the queries and outputs: the HBM traffic of "
                                          "an ideal region-ordered sweep",
                        "traffic": None},
           "with_pvalues": {"ms_per_step": ms_pv, "value": units / (ms_pv / 1e3), "query_length_groups": ngroups,
                            "emitted_cells": emitted, "min_ln_p": min_lp, "moments_build_s": moments_s,
                            "moments": mom_kind,
                            "stage": "query length groups + FP64 p-values of every (file, source) cell on the "
                                     "device (rgl_batch_pvalues_device) after the counts"},
           "e2e": {"value": units / e2e_s, "unit": UNIT, "ms_per_step": e2e_s * 1e3, "h2d_bytes_per_step": N * 12,
                   "d2h_bytes_per_step": F * D * 12, "api": "rgl_query_batch_host (page-locked host intervals)"},
           "cpu_baseline": cpu, "clocks": clk, "l2": "the batch's 5.6 GB of query intervals exceed L2"}
    mom.close()
    ctx.close()
    del t_iv
    if which == "config1":
        idx.close()
    return out


# ---------------------------------------------------------------------------------------------
# serving: Poisson arrivals against the resident 64-file database
# ---------------------------------------------------------------------------------------------
def serve_trace(srv, reqs, arrivals, hp):
    tickets = []
    t0 = time.perf_counter()
    for k, blocks in enumerate(reqs):
        dt = t0 + arrivals[k] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        tickets.append(srv.submit(blocks, intervals_ptr=hp))
    infos = [srv.wait(t, 120_000)[2] for t in tickets]
    return infos


def synthetic_moments(D, cl, file_sizes, device):
    """A moment store for every (source, chromosome) of a synthetic database, with tables of the
    right shape and plausible values (mean = L x the source's mean coverage per bin, variance
    over-dispersed by (1 + L / 100)): the serving and batched stats stages are timed on it.  Their
    cost does not depend on the values; the values themselves are pinned by the p-value tests."""
    from riggle_b200 import api

    nb = (np.asarray(cl, np.uint64) + 99) // 100
    m = api.Moments(D, nb, device=device)
    genome = float(np.sum(cl))
    for c in range(len(cl)):
        L = api.moment_grid(int(nb[c])).astype(np.float64)
        for d in range(D):
            cov = float(file_sizes[d]) * 600.0 / genome  # mean coverage per 100 bp bin
            mv = np.stack([L * cov, L * cov * (1.0 + L / 100.0)], 1).astype(np.float32)
            m.set(d, c, mv)
    return m


def run_serving(args, dev, idx, db_desc, moments=None):
    """Serving at the configured rate, at twice it and at four times it (shorter traces; four times
    is beyond what one file per launch sustains against the 2e9-interval database): continuous
    batching against one query file per launch on the same arrivals."""
    base = serve_once(args, dev, idx, args.serve_rate, args.serve_seconds, 77, db_desc, moments)
    high = serve_once(args, dev, idx, 2 * args.serve_rate, max(1.0, args.serve_seconds / 2.5), 78, db_desc, moments)
    over = serve_once(args, dev, idx, 4 * args.serve_rate, max(1.0, args.serve_seconds / 4), 79, db_desc, moments)
    return dict(base, high_load=high, overload=over)


def serve_once(args, dev, idx, lam, T, seed, db_desc, moments):
    import torch

    import riggle_b200 as rg
    from riggle_b200 import _lib

    lib = rg.load()
    cl = rg.synth_chrom_lengths(1, 24)
    rng = np.random.default_rng(seed)
    arr = np.cumsum(rng.exponential(1.0 / lam, size=int(lam * T * 2) + 64))
    arr = arr[arr < T]
    nreq = len(arr)
    sizes = rg.synth_loguniform_sizes(700 + seed, nreq, 1000, 1_000_000)
    spec = rg.SynthSpec(7000 + seed, cl, sizes)
    off, sh, _ = rg.synth_batch_layout(spec)
    N = int(off[-1])
    t_iv = torch.empty((max(N, 1), 3), dtype=torch.int32, device=f"cuda:{dev}")
    rg.synth_batch_device(spec, off, t_iv.data_ptr(), device=dev)
    if N:
        sort_blocks_device(t_iv, off, dev)  # request files sorted by start, as BED files are
    hp = C.c_void_p()
    _lib.check(lib.rgl_host_alloc(max(N, 1) * 12, C.byref(hp)))
    hv = np.ctypeslib.as_array((C.c_uint32 * (max(N, 1) * 3)).from_address(hp.value))
    hv[:] = t_iv.cpu().numpy().view(np.uint32).reshape(-1)
    del t_iv
    C_ = len(cl)
    reqs = [[(int(sh[b]), int(off[b]), int(off[b + 1])) for b in range(k * C_, (k + 1) * C_) if off[b + 1] > off[b]]
            for k in range(nreq)]

    stats_kw = {"moments": moments, "shard_chrom": np.arange(len(cl), dtype=np.uint32)} if moments else {}

    def measure(**kw):
        srv = rg.Server(idx, **kw, **stats_kw)
        serve_trace(srv, reqs[:32], np.zeros(32), hp.value)  # warm-up burst
        srv.reset_stats()
        infos = serve_trace(srv, reqs, arr, hp.value)
        st = srv.stats()
        srv.close()
        lat = np.array([(i["done_s"] - i["submit_s"]) * 1e3 for i in infos])
        n = np.array([i["intervals"] for i in infos])
        near = lat[(n >= 50_000) & (n <= 200_000)]
        return {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "p999_ms": st["p999_ms"], "max_ms": st["max_ms"],
                "mean_ms": st["mean_ms"],
                "p99_ms_1e5_requests": float(np.percentile(near, 99, method="inverted_cdf")) if len(near) else None,
                "requests_1e5": int(len(near)),
                "sustained_query_intervals_per_s": st["intervals"] / max(1e-9, st["last_done_s"] - st["first_submit_s"]),
                "batches": st["batches"], "mean_batch_requests": st["mean_batch_requests"],
                "workers": st["workers"], "failed": st["failed"], "memory_limited_batches": st["memory_limited"],
                "refused": st["refused"], "workspace_growth_bytes": st["grown_bytes"]}

    batched = measure()
    plain = measure(workers=1, max_batch_requests=1)
    lib.rgl_host_free(hp)
    return {"workload": f"serving: Poisson arrivals at {lam:g}/s for {T:g} s ({nreq} query files, log-uniform "
                        f"[1e3, 1e6] intervals, sorted by start within each chromosome) against the resident "
                        f"{db_desc}; latency = submit to count, overlap "
                        + ("and p-value rows" if moments else "rows") + " in host memory; admission by free device "
                        "memory at batch formation",
            "offered_query_intervals_per_s": float(sizes.sum()) / T, "requests": nreq,
            "continuous_batching": batched, "plain_one_file_per_launch": plain}


# ---------------------------------------------------------------------------------------------
# precision: the FFT sliding-window moments at 2^20-2^26 FFT lengths, FP64 and compensated FP32
# ---------------------------------------------------------------------------------------------
def run_precision(args, dev):
    """Moments of one source's coverage at 64 bp bins on synthetic chromosomes of 2^19..2^25 bins
    (FFT lengths 2^20..2^26), interval density of a config-1 database file (50k intervals per 3.6 Gbp
    genome; 5% broad), with the FP64 and the compensated-FP32 device paths; errors against the oracle's
    exact (double-double, direct) window moments for L in [2^8, 2^16] and the grid's edges, and the
    resulting ln p error of one query file's p-values (oracle compute_analytic_stats fed the device's
    moments vs the exact ones)."""
    import riggle_b200 as rg
    import oracle as O
    from riggle_b200 import api

    sizes = [1 << 19, 1 << 21, 1 << 23, 1 << 25][: max(1, args.precision_sizes)]
    out = []
    for nb in sizes:
        span = nb * 64
        n = max(2000, int(round(50_000 * span / 3.6e9)))
        iv = rg.SynthSpec(31 + nb.bit_length(), np.array([span], np.uint32), [n], broad_fraction=0.05).block(0, 0)
        g = O.depth_signal(iv[:, 0], iv[:, 1], nb, 64)
        grid = O.moment_grid(nb)
        mid = np.nonzero((grid >= 256) & (grid <= 65_536))[0]
        sel = np.unique(np.concatenate([mid[:: max(1, len(mid) // 20)], [0, 10, 99, len(grid) - 1]]))
        t0 = time.perf_counter()
        em, ev = O.moments_exact(g, grid[sel], threads=0)
        oracle_s = time.perf_counter() - t0
        q = rg.SynthSpec(77 + nb.bit_length(), np.array([span], np.uint32), [4000]).block(0, 0)
        groups = [(0, O.query_groups(q[:, 0], q[:, 1], 64))]
        exact_tab = np.zeros((len(grid), 2), np.float32)
        row = {"n_bins": nb, "fft_len": 1 << (2 * nb - 1).bit_length(), "bin_size": 64, "intervals": n,
               "grid_entries": int(len(grid)), "checked_L": int(len(sel)), "oracle_s": oracle_s}
        scale = np.maximum(np.abs(ev), 1e-12 * em * em + 1e-300)
        if nb <= (1 << 21):  # the reference's own f64 formula (the oracle's restatement) beside them
            _, rm, rv = O.moments_from_signal(g)
            row["reference_formula_f64"] = {"max_rel_err_var": float(np.max(np.abs(rv[sel] - ev) / scale)),
                                            "max_rel_err_mean": float(np.max(np.abs(rm[sel] - em) /
                                                                             np.maximum(np.abs(em), 1e-300)))}
        for prec in ("fp64", "fp32c"):
            m = api.Moments(1, [nb], device=dev)
            m.build(0, 0, iv, bin_size=64, report=False, precision=prec)  # warm-up (workspace, twiddles)
            ts = []
            for _ in range(2):
                t0 = time.perf_counter()
                mean, var = m.build(0, 0, iv, bin_size=64, report=True, precision=prec)
                ts.append(time.perf_counter() - t0)
            ev_rel = np.abs(var[sel] - ev) / scale
            em_rel = np.abs(mean[sel] - em) / np.maximum(np.abs(em), 1e-300)
            # ln p of one query file against this source: device moments vs exact ones at the checked L
            tab = np.stack([mean, var], 1).astype(np.float32)
            ex = tab.copy()
            ex[sel] = np.stack([em, ev], 1).astype(np.float32)
            lp_err = None
            w_dev = O.analytic_stats(groups, {0: (nb, tab)}, 200.0)
            w_ex = O.analytic_stats(groups, {0: (nb, ex)}, 200.0)
            if w_dev and w_ex and w_dev[1] is not None and w_ex[1] is not None:
                lp_d = O.lib().orc_log_p(w_dev[1], 1, 1.0, 1.0)
                lp_e = O.lib().orc_log_p(w_ex[1], 1, 1.0, 1.0)
                lp_err = abs(lp_d - lp_e) / max(abs(lp_e), 1e-300)
            row[prec] = {"build_ms": 1e3 * min(ts), "max_rel_err_mean": float(em_rel.max()),
                         "max_rel_err_var": float(ev_rel.max()), "ln_p_rel_err": lp_err,
                         "within_1e-6": bool(em_rel.max() < 1e-6 and ev_rel.max() < 1e-6)}
            m.close()
        out.append(row)
    return {"workload": "config 3: one source's coverage at 64 bp bins, 2^19..2^25 bins (FFT 2^20..2^26), "
                        "config-1 interval density; errors vs the oracle's exact window moments for L in "
                        "[2^8, 2^16] (every ~20th grid L) and the grid's edges",
            "fp64": "FP64 Stockham FFT, double-double prefix sums",
            "fp32c": "compensated FP32: float-float FFT / power spectrum / prefix sums, FP64 only in the final "
                     "per-L reduction and the variance subtraction",
            "sizes": out}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    dist = False
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = True
    big = None
    try:
        out = None
        if args.only in ("all", "plain"):
            out, big = run_riggle(args, rank, world, local_rank, dist)
        if rank == 0 and world == 1 and args.only != "plain":
            import riggle_b200 as rg

            def stub(part, v, unit, hib):
                return {"metric": METRIC, "value": v, "unit": unit, "n_gpus": 1, "higher_is_better": hib,
                        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
                        "config": {"workload": part}}

            if big is None and args.only in ("all", "batched", "serving") and (
                    args.only != "batched" or args.batch_db != "config1"):
                cl, db, _, _ = workload_spec("plain", args.db_intervals, args.chroms)
                big = (rg.Index.synth(db, device=local_rank), db)
            if args.batch_files and args.only in ("all", "batched"):
                if args.batch_db in ("both", "config1"):
                    b = run_batched(args, local_rank, "config1")
                    out = out or stub(b["workload"], b["value"], UNIT, True)
                    out["batched"] = b
                if args.batch_db in ("both", "config2"):
                    b = run_batched(args, local_rank, "config2", big)
                    out = out or stub(b["workload"], b["value"], UNIT, True)
                    out["batched_2e9"] = b
            if args.serve_seconds and args.only in ("all", "serving"):
                idx, db = big
                cl = np.asarray(db.chrom_len)
                mom = synthetic_moments(idx.num_sources, cl, db.file_sizes, local_rank)
                db_desc = f"1,000-file database of {int(np.sum(db.file_sizes)):.3g} intervals (config 2, 24 GB)"
                sv = run_serving(args, local_rank, idx, db_desc, mom)
                mom.close()
                out = out or stub(sv["workload"], sv["continuous_batching"]["p99_ms"], "ms (p99)", False)
                out["serving"] = sv
            if args.precision_sizes and args.only in ("all", "precision"):
                pr = run_precision(args, local_rank)
                out = out or stub(pr["workload"], None, "relative error", False)
                out["precision"] = pr
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if big is not None:
            big[0].close()
        if dist:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
