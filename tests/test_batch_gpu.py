"""The batched form (rgl_query_batch_device): many query files in one call, cut into sub-batches,
optionally captured as one CUDA graph, with the autotuned launch shape.  Every result must equal the
oracle's (and so the one-file-per-call path's) bit for bit.  Needs a GPU."""
import numpy as np
import pytest

import helpers
import oracle as O
import riggle_b200 as rg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(a):
    """uint32 numpy array -> device tensor (kept alive by the caller) and its pointer."""
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to("cuda:0")
    return t, t.data_ptr()


def _file_major(files, nshards):
    """files: list of {shard: uint32[n,3] with sid = file row}.  Returns (intervals, shards, offsets, rows)."""
    parts, shards, offs, rows = [], [], [0], []
    for f, per in enumerate(files):
        for sh in range(nshards):
            a = per.get(sh)
            if a is None or not len(a):
                continue
            parts.append(a)
            shards.append(sh)
            rows.append(f)
            offs.append(offs[-1] + len(a))
    iv = np.concatenate(parts) if parts else np.zeros((0, 3), np.uint32)
    return iv, np.array(shards, np.uint32), np.array(offs, np.uint64), np.array(rows, np.uint32)


def _random_batch(seed, nfiles=37, nshards=3, D=23):
    rng = np.random.default_rng(seed)
    blocks = [(sh, helpers.random_db(rng, int(rng.integers(2000, 20000)), 3_000_000, D)) for sh in range(nshards)]
    layers = rg.bucket_layers(blocks)
    files = []
    for f in range(nfiles):
        per = {}
        for sh, b in blocks:
            n = int(rng.integers(0, 400))
            if n == 0:
                continue
            q = np.concatenate([helpers.queries_touching(rng, b, n, 1), helpers.random_db(rng, n, 3_000_000, 1)])
            q[:, 2] = f
            per[sh] = q
        files.append(per)
    return layers, files, D, nshards


def _oracle(layers, files, D, nshards):
    qsh = {}
    for per in files:
        for sh, a in per.items():
            qsh.setdefault(sh, []).append(a)
    qsh = {k: np.concatenate(v) for k, v in qsh.items()}
    oc, _, obp, _ = O.query_database(layers, qsh, len(files), D, threads=4)
    return oc, obp


def _run(ctx, batch, D, **kw):
    R = batch.num_rows
    dc = torch.empty((R, D), dtype=torch.int32, device="cuda:0")
    db = torch.empty((R, D), dtype=torch.int64, device="cuda:0")
    st = ctx.query_batch_device(batch, dc.data_ptr(), db.data_ptr(), **kw)
    torch.cuda.synchronize()
    return dc.cpu().numpy().view(np.uint32), db.cpu().numpy().view(np.uint64), st


@pytest.mark.parametrize("seed", [1, 2])
def test_batch_matches_oracle_any_sub_batch(seed):
    layers, files, D, nsh = _random_batch(seed)
    oc, obp = _oracle(layers, files, D, nsh)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    t, p = _dev(iv)
    for with_rows in (True, False):
        b = rg.DeviceBatch(len(files), shards, offs, p, rows if with_rows else None)
        # sub-batches that cut blocks and rows in the middle, one sub-batch, and the default
        for sub in (997, 5000, len(iv), 0):
            c, bp, st = _run(ctx, b, D, sub_batch=sub)
            assert (c == oc).all() and (bp == obp).all(), (with_rows, sub)
            assert st["query_intervals"] == len(iv)
            want = -(-len(iv) // sub) if sub else 1
            assert st["sub_batches"] == want
    # the plain one-call path agrees, and so does the batch's swept count with its per-row sum
    ctx.close()
    idx.close()


def test_batch_graph_replay_and_invalidation():
    layers, files, D, nsh = _random_batch(5)
    oc, obp = _oracle(layers, files, D, nsh)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    t, p = _dev(iv)
    b = rg.DeviceBatch(len(files), shards, offs, p, rows)
    R = len(files)
    dc = torch.empty((R, D), dtype=torch.int32, device="cuda:0")
    dbp = torch.empty((R, D), dtype=torch.int64, device="cuda:0")

    def run(**kw):
        st = ctx.query_batch_device(b, dc.data_ptr(), dbp.data_ptr(), graph=True, sub_batch=3000, **kw)
        return dc.cpu().numpy().view(np.uint32), dbp.cpu().numpy().view(np.uint64), st

    c, bp, st = run()
    assert st["graph_replayed"] == 0 and st["graph_nodes"] > 0
    assert (c == oc).all() and (bp == obp).all()
    dc.fill_(7)
    c, bp, st = run()
    assert st["graph_replayed"] == 1
    assert (c == oc).all() and (bp == obp).all()
    # new interval values in the same buffer and layout: the replay reads them at launch
    iv2 = iv.copy()
    iv2[:, 0] //= 2
    t.copy_(torch.from_numpy(iv2.view(np.int32)))
    files2 = []
    at = 0
    for per in files:
        d = {}
        for sh in range(nsh):
            if sh in per and len(per[sh]):
                d[sh] = iv2[at:at + len(per[sh])]
                at += len(per[sh])
        files2.append(d)
    oc2, obp2 = _oracle(layers, files2, D, nsh)
    c, bp, st = run()
    assert st["graph_replayed"] == 1
    assert (c == oc2).all() and (bp == obp2).all()
    # a plain call that grows the workspace invalidates the graph: the next batch call recaptures
    big = np.concatenate([a for per in files2 for a in per.values()] * 3)
    big[:, 2] = 0
    ctx.query_counts({"s0": big}, 1)
    c, bp, st = run()
    assert st["graph_replayed"] == 0
    assert (c == oc2).all() and (bp == obp2).all()
    # a different launch shape is a different graph
    c, bp, st = run(chunk=512)
    assert st["graph_replayed"] == 0 and st["chunk"] == 512
    assert (c == oc2).all() and (bp == obp2).all()
    ctx.close()
    idx.close()


def test_batch_autotune_and_tuned_shape():
    layers, files, D, nsh = _random_batch(7)
    oc, obp = _oracle(layers, files, D, nsh)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    t, p = _dev(iv)
    b = rg.DeviceBatch(len(files), shards, offs, p, rows)
    best, trials = ctx.autotune(b, sub_batch=4000)
    assert len(trials) == 4 + 25
    assert best["chunk"] in (512, 1024, 2048, 4096, 8192) and best["ctas_per_sm"] in (2, 3, 4, 6, 8)
    assert best["pair_ratio"] in (1, 2, 4, 8)
    assert min(tr["sweep_ms"] for tr in trials) > 0
    c, bp, st = _run(ctx, b, D, tuned=True, graph=True)
    assert (c == oc).all() and (bp == obp).all()
    assert (st["chunk"], st["ctas_per_sm"], st["pair_ratio"]) == (best["chunk"], best["ctas_per_sm"],
                                                                    best["pair_ratio"])
    ctx.close()
    idx.close()


def test_batch_errors_and_empty():
    layers, files, D, nsh = _random_batch(3, nfiles=5)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    # empty batch: zero outputs
    b0 = rg.DeviceBatch(5, np.zeros(0, np.uint32), np.zeros(1, np.uint64), 0)
    c, bp, st = _run(ctx, b0, D)
    assert (c == 0).all() and (bp == 0).all() and st["query_intervals"] == 0
    # an interval whose sid is outside its block's row
    bad = iv.copy()
    bad[len(bad) // 2, 2] = (bad[len(bad) // 2, 2] + 1) % 5  # a valid row, not its block's
    t, p = _dev(bad)
    b = rg.DeviceBatch(5, shards, offs, p, rows)
    with pytest.raises(rg.RiggleError, match="INVALID_ARGUMENT"):
        _run(ctx, b, D, sub_batch=50)
    # asynchronous form: the error is reported by the context check
    dc = torch.empty((5, D), dtype=torch.int32, device="cuda:0")
    ctx.query_batch_device(b, dc.data_ptr(), None, stats=False)
    with pytest.raises(rg.RiggleError, match="INVALID_ARGUMENT"):
        ctx.check()
    # start >= end
    bad2 = iv.copy()
    bad2[0, 1] = bad2[0, 0]
    t2, p2 = _dev(bad2)
    with pytest.raises(rg.RiggleError, match="INVALID_ARGUMENT"):
        _run(ctx, rg.DeviceBatch(5, shards, offs, p2, rows), D)
    # host-side checks
    with pytest.raises(rg.RiggleError, match="shard id"):
        _run(ctx, rg.DeviceBatch(5, shards + 7, offs, p, rows), D)
    with pytest.raises(rg.RiggleError, match="row"):
        _run(ctx, rg.DeviceBatch(5, shards, offs, p, rows + 9), D)
    # the context stays usable
    t3, p3 = _dev(iv)
    oc, obp = _oracle(layers, files, D, nsh)
    c, bp, _ = _run(ctx, rg.DeviceBatch(5, shards, offs, p3, rows), D)
    assert (c == oc).all() and (bp == obp).all()
    ctx.close()
    idx.close()


def test_device_batch_generator_matches_host_blocks():
    cl = rg.synth_chrom_lengths(1, 24)
    sizes = rg.synth_loguniform_sizes(4, 6, 100, 30000)
    spec = rg.SynthSpec(4000, cl, sizes, hotspot_fraction=0.1, num_hotspots=8)
    off, sh, rw = rg.synth_batch_layout(spec)
    assert int(off[-1]) == int(sizes.sum())
    t = torch.empty((int(off[-1]), 3), dtype=torch.int32, device="cuda:0")
    rg.synth_batch_device(spec, off, t.data_ptr())
    dev = t.cpu().numpy().view(np.uint32)
    for f in range(spec.num_files):
        for c in range(spec.num_chroms):
            b = f * spec.num_chroms + c
            assert sh[b] == c and rw[b] == f
            got = dev[int(off[b]):int(off[b + 1])]
            want = spec.block(f, c)
            key = lambda a: a[np.lexsort((a[:, 2], a[:, 1], a[:, 0]))]
            assert (key(got) == key(want)).all(), (f, c)


def test_config1_database_batch_equals_one_file_per_call():
    """Config-1 database (64 files x 50k) against a batch of hot-spot query files: the batched form
    equals the plain one-file-per-call form on every row."""
    cl = rg.synth_chrom_lengths(1, 24)
    db = rg.Index.synth(rg.SynthSpec(2, cl, np.full(64, 50_000, np.uint64)))
    sizes = rg.synth_loguniform_sizes(11, 24, 100, 100_000)
    spec = rg.SynthSpec(1000, cl, sizes, hotspot_fraction=0.1, num_hotspots=8)
    off, sh, rw = rg.synth_batch_layout(spec)
    t = torch.empty((int(off[-1]), 3), dtype=torch.int32, device="cuda:0")
    rg.synth_batch_device(spec, off, t.data_ptr())
    ctx = rg.Context(db)
    b = rg.DeviceBatch(spec.num_files, sh, off, t.data_ptr(), rw)
    c, bp, _ = _run(ctx, b, 64, sub_batch=1 << 18, graph=True)
    # the swept count of the per-file unions: the region work order adds boundary windows to it
    _, _, st = _run(ctx, b, 64, sub_batch=1 << 18, region_bits=rg._lib.RGL_BATCH_NO_REGIONS)
    host = t.cpu().numpy().view(np.uint32)
    swept = 0
    for f in range(spec.num_files):
        per = {}
        for ch in range(spec.num_chroms):
            k = f * spec.num_chroms + ch
            a = host[int(off[k]):int(off[k + 1])].copy()
            if len(a):
                a[:, 2] = 0
                per[int(ch)] = a
        pc, pbp, pst = ctx.query_counts(per, 1)
        assert (c[f] == pc[0]).all() and (bp[f] == pbp[0]).all(), f
        swept += pst["db_swept"]
    assert st["db_swept"] == swept
    ctx.close()
    db.close()


def test_large_and_small_runs_agree():
    """Runs above 2^21 query intervals launch the pipeline's short kernels without programmatic
    dependent launch, smaller runs with it; one batch of ~6M intervals as one run and as runs of
    2^20 must agree on every cell (and the large run must take the block-local sort for no block:
    these files have blocks above 16,384 intervals)."""
    cl = rg.synth_chrom_lengths(1, 24)
    db = rg.Index.synth(rg.SynthSpec(2, cl, np.full(64, 50_000, np.uint64)))
    sizes = rg.synth_loguniform_sizes(17, 12, 100_000, 1_000_000)
    spec = rg.SynthSpec(3000, cl, sizes, hotspot_fraction=0.1, num_hotspots=8)
    off, sh, rw = rg.synth_batch_layout(spec)
    assert int(off[-1]) > (1 << 21) and int(np.diff(off).max()) > 16384
    t = torch.empty((int(off[-1]), 3), dtype=torch.int32, device="cuda:0")
    rg.synth_batch_device(spec, off, t.data_ptr())
    ctx = rg.Context(db)
    b = rg.DeviceBatch(spec.num_files, sh, off, t.data_ptr(), rw)
    c1, bp1, st1 = _run(ctx, b, 64, sub_batch=int(off[-1]))
    c2, bp2, st2 = _run(ctx, b, 64, sub_batch=1 << 20)
    assert st1["sub_batches"] == 1 and st2["sub_batches"] > 1
    assert (c1 == c2).all() and (bp1 == bp2).all()
    assert c1.sum() > 0
    ctx.close()
    db.close()


def test_host_batch_pipelined_copies_equal_device_batch():
    layers, files, D, nsh = _random_batch(13, nfiles=29)
    oc, obp = _oracle(layers, files, D, nsh)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    b = rg.DeviceBatch(len(files), shards, offs, 0, rows)
    for sub in (1009, 4000, 0):  # several sub-batches alternate the two staging buffers
        c, bp, st = ctx.query_batch_host(b, iv, sub_batch=sub)
        assert (c == oc).all() and (bp == obp).all(), sub
        assert st["query_intervals"] == len(iv)
    c, bp, st = ctx.query_batch_host(b, iv, with_overlap=False, sub_batch=3000)
    assert (c == oc).all() and bp is None
    # an error in one sub-batch is reported and leaves the context usable
    bad = iv.copy()
    bad[-1, 1] = bad[-1, 0]
    with pytest.raises(rg.RiggleError, match="INVALID_ARGUMENT"):
        ctx.query_batch_host(b, bad, sub_batch=2000)
    c, bp, _ = ctx.query_batch_host(b, iv, sub_batch=2000)
    assert (c == oc).all() and (bp == obp).all()
    ctx.close()
    idx.close()


@pytest.mark.parametrize("seed", [21, 22])
def test_batch_pvalues_device_equal_host_stats_path(seed):
    """The batch's stats stage on the device (length groups built from the batch's intervals) equals
    the host path (rgl_query_chrom_groups per row and chromosome + rgl_query_pvalues), which the
    p-value tests pin to the oracle."""
    from riggle_b200 import api

    rng = np.random.default_rng(seed)
    layers, files, D, nsh = _random_batch(seed, nfiles=23, nshards=3, D=11)
    nbins = [30_001, 25_000, 7]  # chromosome 2 is tiny: most of its groups have l_int >= n_bins
    m = api.Moments(D, nbins)
    tables = {}
    for d in range(D):
        for c in range(len(nbins)):
            if rng.random() < 0.2:
                continue
            ns = m.slots(c)
            mean = np.sort(rng.random(ns) * rng.uniform(0.01, 50))
            var = mean * (rng.uniform(1.5, 30) if rng.random() < 0.6 else rng.uniform(0.1, 0.9))
            mv = np.stack([mean, var], 1).astype(np.float32)
            mv = mv[: ns // 2] if rng.random() < 0.1 else mv
            m.set(d, c, mv)
            tables[(d, c)] = mv
    shard_chrom = np.array([0, 1, 0xFFFFFFFF if seed % 2 else 2], np.uint32)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    t, p = _dev(iv)
    b = rg.DeviceBatch(len(files), shards, offs, p, rows)
    R = len(files)
    dc = torch.empty((R, D), dtype=torch.int32, device="cuda:0")
    dbp = torch.empty((R, D), dtype=torch.int64, device="cuda:0")
    ctx.query_batch_device(b, dc.data_ptr(), dbp.data_ptr(), sub_batch=3000)
    out = {k: torch.empty((R, D), dtype=dt, device="cuda:0")
           for k, dt in (("p", torch.float64), ("llr", torch.float64), ("lp", torch.float64), ("f", torch.uint8))}
    ng = m.batch_pvalues_device(ctx, b, shard_chrom, dc.data_ptr(), dbp.data_ptr(), out["p"].data_ptr(),
                                out["llr"].data_ptr(), out["lp"].data_ptr(), out["f"].data_ptr())
    torch.cuda.synchronize()
    assert ng > 0
    counts = dc.cpu().numpy().view(np.uint32)
    bp = dbp.cpu().numpy().view(np.uint64)
    # the oracle's own groups (its restatement of build_query_chrom_data) on the reference side
    row_groups = []
    for per in files:
        chroms = []
        for sh, a in sorted(per.items()):
            if shard_chrom[sh] != 0xFFFFFFFF:
                chroms.append((int(shard_chrom[sh]), O.query_groups(a[:, 0], a[:, 1])))
        row_groups.append(chroms)
    hp, hl, hlp, hf = m.pvalues(row_groups, counts, bp)
    dp, dl, dlp, df = (out[k].cpu().numpy() for k in ("p", "llr", "lp", "f"))
    assert (df == hf).all()
    assert (hf & 1).sum() > 10  # emitted cells exist
    np.testing.assert_allclose(dl, hl, rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(dp, hp, rtol=1e-11, atol=1e-300)
    np.testing.assert_allclose(dlp, hlp, rtol=1e-11, atol=1e-13)
    # and every emitted cell against the oracle's compute_analytic_stats directly
    checked = 0
    for q in range(R):
        for d in range(D):
            if not counts[q, d]:
                continue
            db = {c: (nbins[c], tables[(d, c)]) for c in range(len(nbins)) if (d, c) in tables}
            want = O.analytic_stats(row_groups[q], db, float(bp[q, d]) / 100.0)
            if want is None:
                assert df[q, d] == 0
                continue
            wp, wl = want
            assert df[q, d] & 1 and bool(df[q, d] & 2) == (wl is not None)
            if wl is not None:
                assert dl[q, d] == pytest.approx(wl, rel=1e-9, abs=1e-12)
            assert dp[q, d] == pytest.approx(wp, rel=1e-9, abs=1e-300)
            checked += 1
    assert checked > 10
    ctx.close()
    m.close()
    idx.close()


@pytest.mark.parametrize("seed", [11, 12])
def test_work_order_and_tally_modes_agree_with_the_oracle(seed):
    """The region work order (every row's work on a 2^k-bp region laid out together) and the
    block-local histograms of several-row sweeps change only the order of additions: every combination
    (regions of 64 kbp, 16 Mbp, none; shared-memory or global tallies; chunk sizes that put many rows in
    one block item) gives the oracle's counts and base pairs bit for bit."""
    layers, files, D, nsh = _random_batch(seed, nfiles=29)
    oc, obp = _oracle(layers, files, D, nsh)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    iv, shards, offs, rows = _file_major(files, nsh)
    t, p = _dev(iv)
    b = rg.DeviceBatch(len(files), shards, offs, p, rows)
    swept = {}
    for rb in (16, 24, rg._lib.RGL_BATCH_NO_REGIONS):
        for tally in ("shared", "global"):
            for chunk in (0, 128):
                c, bp, st = _run(ctx, b, D, region_bits=rb, global_tally=tally == "global", chunk=chunk,
                                 sub_batch=4000)
                assert (c == oc).all() and (bp == obp).all(), (rb, tally, chunk)
                swept[rb] = st["db_swept"]
    # counts only (no overlap): the 32-bit shared histogram of the row
    c, _, _ = _run(ctx, b, D, counts_only=True, sub_batch=4000)
    assert (c == oc).all()
    # regions can only add look-back windows that cross region boundaries to the swept count
    assert swept[16] >= swept[24] >= swept[rg._lib.RGL_BATCH_NO_REGIONS]
    ctx.close()
    idx.close()


def test_batch_blocks_in_any_order_and_of_many_tiles():
    """Blocks handed over in a shuffled order (rows and shards interleaved), some of them several
    sort tiles long, some already sorted by start: the block-local key sort lays the keys out in
    segment order and must give the oracle's counts and overlaps, in one sub-batch and in several."""
    rng = np.random.default_rng(21)
    D, nsh = 19, 3
    dbs = [(sh, helpers.random_db(rng, int(rng.integers(5000, 20000)), 3_000_000, D)) for sh in range(nsh)]
    layers = rg.bucket_layers(dbs)
    files = []
    for f in range(9):
        per = {}
        for sh, b in dbs:
            n = int(rng.choice([0, 50, 4096, 4097, 9000, 20000]))
            if n == 0:
                continue
            q = np.concatenate([helpers.queries_touching(rng, b, n // 2, 1), helpers.random_db(rng, n - n // 2, 3_000_000, 1)])
            if rng.random() < 0.5:
                q = q[np.lexsort((q[:, 1], q[:, 0]))]
            q[:, 2] = f
            per[sh] = q
        files.append(per)
    oc, obp = _oracle(layers, files, D, nsh)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    keys = [(f, sh) for f, per in enumerate(files) for sh in per]
    order = [keys[k] for k in rng.permutation(len(keys))]
    parts = [files[f][sh] for f, sh in order]
    offs = np.zeros(len(parts) + 1, np.uint64)
    offs[1:] = np.cumsum([len(a) for a in parts])
    iv = np.concatenate(parts)
    t, p = _dev(iv)
    b = rg.DeviceBatch(len(files), np.array([sh for _, sh in order], np.uint32), offs, p,
                       np.array([f for f, _ in order], np.uint32))
    for sub in (0, 30011):
        c, bp, _ = _run(ctx, b, D, sub_batch=sub)
        assert (c == oc).all() and (bp == obp).all(), sub
    ctx.close()
    idx.close()
