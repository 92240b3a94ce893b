"""Parity of the CUDA sweep (through the C ABI) with the CPU oracle.  Needs a GPU."""
import numpy as np
import pytest

import helpers
import oracle as O
import riggle_b200 as rg
from riggle_b200 import _lib

pytestmark = pytest.mark.gpu


def gpu_counts(layers, qshards, rows, num_sources, nshards, min_size=128, gf=4, **kw):
    idx = rg.Index.from_layers(layers, num_sources, [f"s{i}" for i in range(nshards)], min_size, gf)
    ctx = rg.Context(idx)
    c, bp, st = ctx.query_counts(qshards, rows, **kw)
    ctx.close()
    idx.close()
    return c, bp, st


def test_known_answers(known):
    for case in known["sweep"]:
        db = np.array(case["db"], np.uint32).reshape(-1, 3)
        q = np.array(case["query"], np.uint32).reshape(-1, 3)
        layers = {(0, 0): (db[:, :2], db[:, 2])} if len(db) else {}
        # min_size = the case's layer_max puts every DB interval in layer 0 with that look-back
        c, bp, _ = gpu_counts(layers, {0: q} if len(q) else {}, case["rows"], case["cols"], 1,
                              min_size=case["layer_max"], gf=4)
        assert c.tolist() == case["counts"], case["ref"]
        np.testing.assert_allclose(bp / 100.0, case["bins"], atol=1e-6, err_msg=case["ref"])


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_parity_with_oracle(seed):
    rng = np.random.default_rng(seed)
    rows, D, nsh = int(rng.integers(1, 70)), int(rng.integers(1, 40)), 3
    blocks = [(sh, helpers.random_db(rng, int(rng.integers(100, 20000)), 3_000_000, D)) for sh in range(nsh)]
    layers = rg.bucket_layers(blocks)
    qsh = {}
    for sh, b in blocks:
        q1 = helpers.queries_touching(rng, b, 500, rows)
        q2 = helpers.random_db(rng, 500, 3_000_000, rows)
        qsh[sh] = np.concatenate([q1, q2])
    oc, _, obp, ost = O.query_database(layers, qsh, rows, D, threads=4)
    c, bp, st = gpu_counts(layers, {f"s{k}": v for k, v in qsh.items()}, rows, D, nsh)
    assert (c == oc).all()
    assert (bp == obp).all()
    for ratio in (1, 1000000):  # all ranges by rank differences / all pair by pair
        c2, bp2, _ = gpu_counts(layers, {f"s{k}": v for k, v in qsh.items()}, rows, D, nsh, pair_ratio=ratio)
        assert (c2 == oc).all() and (bp2 == obp).all()
    # the device sweeps the union of candidate ranges once per (shard, query row)
    per_row = 0
    for r in range(rows):
        sub = {k: v[v[:, 2] == r] for k, v in qsh.items()}
        sub = {k: np.concatenate([v[:, :2], np.zeros((len(v), 1), np.uint32)], 1) for k, v in sub.items() if len(v)}
        per_row += O.query_database(layers, sub, 1, D)[3]["db_swept"] if sub else 0
    assert st["db_swept"] == per_row


def test_small_parity_with_bruteforce_u32_extremes():
    rng = np.random.default_rng(9)
    top = 2**32 - 1
    s = rng.integers(top - 5_000_000, top - 3000, 3000).astype(np.int64)
    e = s + rng.integers(1, 3000, 3000)
    db = np.stack([s, e, rng.integers(0, 5, 3000)], 1).astype(np.uint32)
    qs = rng.integers(top - 5_000_000, top - 1, 400).astype(np.int64)
    qe = np.minimum(qs + rng.integers(1, 10000, 400), top)
    q = np.stack([qs, qe, rng.integers(0, 3, 400)], 1).astype(np.uint32)
    q = q[q[:, 0] < q[:, 1]]
    layers = rg.bucket_layers([(0, db)])
    bc, bbp = O.bruteforce(layers, {0: q}, 3, 5)
    c, bp, _ = gpu_counts(layers, {0: q}, 3, 5, 1)
    assert (c == bc).all() and (bp == bbp).all()


def test_counts_only_flag_and_empty_batch():
    rng = np.random.default_rng(4)
    db = helpers.random_db(rng, 5000, 1_000_000, 6)
    layers = rg.bucket_layers([(0, db)])
    q = helpers.random_db(rng, 300, 1_000_000, 2)
    oc, _, _, _ = O.query_database(layers, {0: q}, 2, 6)
    c, bp, _ = gpu_counts(layers, {0: q}, 2, 6, 1, with_overlap=False)
    assert bp is None and (c == oc).all()
    c, bp, st = gpu_counts(layers, {}, 2, 6, 1)
    assert not c.any() and not bp.any() and st["db_swept"] == 0
    # a shard the index does not know is skipped (src/tasks/query/mod.rs:194-196)
    c, bp, _ = gpu_counts(layers, {"chrUnknown": q}, 2, 6, 1)
    assert not c.any()


def test_invalid_query_intervals_are_rejected():
    db = np.array([[10, 20, 0]], np.uint32)
    layers = rg.bucket_layers([(0, db)])
    with pytest.raises(rg.RiggleError) as e:
        gpu_counts(layers, {0: np.array([[30, 30, 0]], np.uint32)}, 1, 1, 1)
    assert e.value.status == _lib.RGL_ERR_INVALID_ARGUMENT
    with pytest.raises(rg.RiggleError) as e:
        gpu_counts(layers, {0: np.array([[5, 30, 4]], np.uint32)}, 2, 1, 1)
    assert e.value.status == _lib.RGL_ERR_INVALID_ARGUMENT


def test_index_rejects_unsorted_layer_and_bad_sid():
    pos = np.array([[50, 60], [10, 20]], np.uint32)
    with pytest.raises(rg.RiggleError) as e:
        rg.Index.from_layers({(0, 0): (pos, np.array([0, 0], np.uint32))}, 1, ["a"])
    assert e.value.status == _lib.RGL_ERR_INDEX_INVARIANT
    pos = np.array([[10, 20], [50, 60]], np.uint32)
    with pytest.raises(rg.RiggleError) as e:
        rg.Index.from_layers({(0, 0): (pos, np.array([0, 3], np.uint32))}, 2, ["a"])
    assert e.value.status == _lib.RGL_ERR_INDEX_INVARIANT


def test_launch_shapes_do_not_change_results():
    rng = np.random.default_rng(12)
    blocks = [(0, helpers.random_db(rng, 30000, 10_000_000, 9))]
    layers = rg.bucket_layers(blocks)
    q = helpers.random_db(rng, 3000, 10_000_000, 1)
    idx = rg.Index.from_layers(layers, 9, ["a"])
    ctx = rg.Context(idx)
    ref = None
    for chunk in (256, 1024, 4096, 16384):
        for cps, ratio in ((1, 1), (2, 4), (4, 0), (8, 1000000)):
            c, bp, _ = ctx.query_counts({0: q}, 1, chunk=chunk, ctas_per_sm=cps, pair_ratio=ratio)
            if ref is None:
                ref = (c, bp)
            assert (c == ref[0]).all() and (bp == ref[1]).all()


def synth_config1(num_files=64, per_file=50_000):
    cl = rg.synth_chrom_lengths(1, 24)
    db = rg.SynthSpec(2, cl, [per_file] * num_files)
    q = rg.SynthSpec(1000, cl, [10_000])
    return cl, db, q


def test_device_synth_index_matches_host_blocks():
    cl = rg.synth_chrom_lengths(1, 24)
    sp = rg.SynthSpec(7, cl, [3000, 5000, 100], broad_fraction=0.05)
    idx = rg.Index.synth(sp)
    blocks = [(c, np.concatenate([sp.block(f, c) for f in range(sp.num_files)])) for c in range(24)]
    host = rg.bucket_layers(blocks)
    for (sh, k), (pos, sid) in host.items():
        dpos, dsid = idx.export_layer(sh, k)
        a = np.concatenate([pos, sid[:, None]], 1)
        b = np.concatenate([dpos, dsid[:, None]], 1)
        a = a[np.lexsort(a.T[::-1])]
        b = b[np.lexsort(b.T[::-1])]
        assert (a == b).all()
        assert (np.diff(dpos[:, 0].astype(np.int64)) >= 0).all()
    assert idx.num_intervals == sum(len(v[1]) for v in host.values())


def test_config1_parity_with_oracle():
    """64 DB files x 50k intervals, one query file of 10k (the CPU-runnable configuration)."""
    cl, dbs, qs = synth_config1()
    idx = rg.Index.synth(dbs)
    layers = {}
    for sh in range(24):
        for k in range(idx.num_layer_slots):
            if idx.layer_count(sh, k):
                layers[(sh, k)] = idx.export_layer(sh, k)
    qsh = {c: qs.block(0, c) for c in range(24)}
    oc, of32, obp, ost = O.query_database(layers, qsh, 1, 64, threads=8)
    ctx = rg.Context(idx)
    c, bp, st = ctx.query_counts({rg.CHROM_NAMES_24[c]: v for c, v in qsh.items()}, 1)
    assert (c == oc).all() and (bp == obp).all()
    assert st["db_swept"] == ost["db_swept"]
    # the reference's f32 bins agree with exact bp / 100 to f32 accumulation error
    np.testing.assert_allclose(of32, obp / 100.0, rtol=1e-4)


def test_block_local_sort_equals_radix_sort():
    """With one row and one block per chromosome, the keys are sorted block by block: tiles of
    4,096 intervals in shared memory (copied through when a block is already in order), then merge
    passes for larger blocks; with a chromosome in two blocks, by the device-wide radix sort.  Both
    must give the oracle's counts and overlaps: unsorted blocks, sorted ones (starts in order, ends
    not), blocks of 1 to 35 tiles (0 to 6 merge passes, blocks of different pass counts in one run),
    equal starts and whole duplicates."""
    rng = np.random.default_rng(11)
    D = 23
    blocks = [(sh, helpers.random_db(rng, 30000, 2_000_000, D)) for sh in range(2)]
    layers = rg.bucket_layers(blocks)

    def queries(b, n):
        q = np.concatenate([helpers.queries_touching(rng, b, n // 2, 1), helpers.random_db(rng, n - n // 2, 2_000_000, 1)])
        q[:, 2] = 0
        q[: n // 8] = q[n // 8: 2 * (n // 8)]  # equal starts (and whole duplicates)
        return q[rng.permutation(n)]

    idx = rg.Index.from_layers(layers, D, ["s0", "s1"])
    ctx = rg.Context(idx)
    cases = ((5000, 700, False, False), (16384, 3000, True, False), (16384, 16385, False, False),
             (40000, 16385, False, True), (70001, 33000, True, False), (140000, 50000, False, True))
    for n0, n1, sort0, sort1 in cases:
        q0, q1 = queries(blocks[0][1], n0), queries(blocks[1][1], n1)
        if sort0:
            q0 = q0[np.lexsort((q0[:, 1], q0[:, 0]))]
        if sort1:
            q1 = q1[np.lexsort((q1[:, 1], q1[:, 0]))]
        oc, _, obp, _ = O.query_database(layers, {0: q0.copy(), 1: q1.copy()}, 1, D, threads=4)
        local = ctx.query_counts({"s0": q0, "s1": q1}, 1)  # one block per chromosome
        k = n0 // 3
        split = ctx.query_counts({"s0": q0[:k], 0: q0[k:], "s1": q1}, 1)  # chromosome 0 in two blocks
        for c, bp, _ in (local, split):
            assert (c == oc).all() and (bp == obp).all(), (n0, n1, sort0, sort1)
