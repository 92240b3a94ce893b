"""Column sharding of the database across ranks: the partition, the host-side column filter and
the all-gather of column slices, as two gloo ranks on the CPU (the oracle answers each rank's
shard), plus the device column filter on one GPU."""
import os
import socket

import numpy as np
import pytest

import helpers
import oracle as O
import riggle_b200 as rg
from riggle_b200 import sharding


def test_column_bounds_partition():
    rng = np.random.default_rng(3)
    for _ in range(50):
        n = int(rng.integers(1, 60))
        parts = int(rng.integers(1, 10))
        sizes = rng.integers(1, 1000, n)
        b = sharding.column_bounds(sizes, parts)
        assert len(b) == parts + 1 and b[0] == 0 and b[-1] == n
        assert (np.diff(b) >= 0).all()
        if parts <= n:
            assert (np.diff(b) >= 1).all()  # every rank owns at least one source
    # balance: with many small sources every share is within one source of the mean
    sizes = np.full(1000, 7)
    b = sharding.column_bounds(sizes, 8)
    share = np.add.reduceat(sizes, b[:-1])
    assert share.max() - share.min() <= 7
    assert list(sharding.column_bounds([100, 1, 1, 1, 1], 2)) == [0, 1, 5]  # one big file alone
    zipf = (np.arange(1, 1001) ** -1.1 * 1e7).astype(np.int64)
    b = sharding.column_bounds(zipf, 4)
    share = np.add.reduceat(zipf, b[:-1])
    assert share.max() - share.min() <= zipf[b[1] - 1]


def _case(seed):
    rng = np.random.default_rng(seed)
    D, nsh, rows = 13, 3, 5
    blocks = [(sh, helpers.random_db(rng, int(rng.integers(2000, 8000)), 2_000_000, D)) for sh in range(nsh)]
    layers = rg.bucket_layers(blocks)
    q = {sh: np.concatenate([helpers.queries_touching(rng, b, 300, rows), helpers.random_db(rng, 300, 2_000_000, rows)])
         for sh, b in blocks}
    sizes = np.bincount(np.concatenate([s for _, s in layers.values()]), minlength=D)
    return layers, q, rows, D, sizes


def _rank_main(rank, world, port, seed):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        layers, q, rows, D, sizes = _case(seed)
        b = sharding.column_bounds(sizes, world)
        mine = sharding.host_layers_columns(layers, int(b[rank]), int(b[rank + 1]))
        width = int(b[rank + 1] - b[rank])
        if mine:
            c, _, bp, _ = O.query_database(mine, {k: v.copy() for k, v in q.items()}, rows, width)
        else:
            c, bp = np.zeros((rows, width), np.uint32), np.zeros((rows, width), np.uint64)
        full_c = sharding.gather_columns(torch.from_numpy(c.view(np.int32)), b)
        full_bp = sharding.gather_columns(torch.from_numpy(bp.view(np.int64)), b)
        oc, _, obp, _ = O.query_database(layers, {k: v.copy() for k, v in q.items()}, rows, D)
        assert (full_c.numpy().view(np.uint32) == oc).all()
        assert (full_bp.numpy().view(np.uint64) == obp).all()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("seed", [1, 2])
def test_two_rank_column_shards_gather_to_the_full_matrix(seed):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(2, _free_port(), seed), nprocs=2, join=True)


@pytest.mark.gpu
def test_device_column_filter_equals_full_columns():
    layers, q, rows, D, sizes = _case(7)
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(3)])
    ctx = rg.Context(idx)
    full_c, full_bp, _ = ctx.query_counts({f"s{k}": v for k, v in q.items()}, rows)
    b = sharding.column_bounds(sizes, 3)
    for r in range(3):
        sub = idx.select_columns(int(b[r]), int(b[r + 1]))
        assert sub.num_sources == b[r + 1] - b[r]
        host = sharding.host_layers_columns(layers, int(b[r]), int(b[r + 1]))
        for (sh, k), (pos, sid) in host.items():  # the device filter keeps order and rebases sids
            p2, s2 = sub.export_layer(sh, k)
            assert (p2 == pos).all() and (s2 == sid).all()
        sctx = rg.Context(sub)
        c, bp, _ = sctx.query_counts({f"s{k}": v for k, v in q.items()}, rows)
        assert (c == full_c[:, b[r]:b[r + 1]]).all() and (bp == full_bp[:, b[r]:b[r + 1]]).all()
        sctx.close()
        sub.close()
    ctx.close()
    idx.close()


@pytest.mark.gpu
def test_synth_columns_equal_select_columns():
    cl = rg.synth_chrom_lengths(1, 4)
    spec = rg.SynthSpec(2, cl, rg.synth_zipf_sizes(12, 1.1, 100, 20000, 60000), broad_fraction=0.05)
    full = rg.Index.synth(spec)
    for lo, hi in ((0, 1), (1, 5), (5, 12)):
        a = rg.Index.synth_columns(spec, lo, hi)
        b = full.select_columns(lo, hi)
        assert a.num_intervals == b.num_intervals and a.num_sources == hi - lo
        assert a.source_name(0) == f"source_{lo}.bed"
        for sh in range(4):
            for k in range(full.num_layer_slots):
                pa, sa = a.export_layer(sh, k)
                pb, sb = b.export_layer(sh, k)
                # same multiset per layer (ties in start may order differently)
                ka = np.lexsort((sa, pa[:, 1], pa[:, 0]))
                kb = np.lexsort((sb, pb[:, 1], pb[:, 0]))
                assert (pa[ka] == pb[kb]).all() and (sa[ka] == sb[kb]).all()
        a.close()
        b.close()
    full.close()
