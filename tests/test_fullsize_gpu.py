"""Parity at the full GPU-scale size: the 1,000-file Zipf database of 2e9 intervals (5% broad) and a
1e5-interval query file, checked through properties that do not depend on size and against the
oracle on one full-density chromosome.  Needs a GPU with ~40 GB free."""
import os

import numpy as np
import pytest

import oracle as O
import riggle_b200 as rg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def full():
    cl = rg.synth_chrom_lengths(1, 24)
    sizes = rg.synth_zipf_sizes(1000, 1.1, 1000, 10_000_000, 2_000_000_000)
    spec = rg.SynthSpec(2, cl, sizes, broad_fraction=0.05)
    idx = rg.Index.synth(spec)
    ctx = rg.Context(idx)
    q = rg.SynthSpec(1234, cl, [100_000])
    qsh = {rg.CHROM_NAMES_24[c]: q.block(0, c) for c in range(24)}
    yield cl, spec, idx, ctx, qsh
    ctx.close()
    idx.close()


def test_pair_scan_rank_differences_and_hybrid_agree(full):
    cl, spec, idx, ctx, qsh = full
    c_h, bp_h, st = ctx.query_counts(qsh, 1)
    assert idx.num_intervals == 2_000_000_000 and st["db_swept"] > 1e8
    assert st["rank_positions"] > 0 and st["pair_candidates"] > 0  # both sweeps take part
    c_p, bp_p, st_p = ctx.query_counts(qsh, 1, pair_ratio=1_000_000)  # every range pair by pair
    assert st_p["rank_positions"] == 0
    assert (c_p == c_h).all() and (bp_p == bp_h).all()
    c_r, bp_r, st_r = ctx.query_counts(qsh, 1, pair_ratio=1)  # more ranges by rank differences
    assert st_r["rank_positions"] > st["rank_positions"]
    assert (c_r == c_h).all() and (bp_r == bp_h).all()
    c_c, _, _ = ctx.query_counts(qsh, 1, with_overlap=False)  # counts-only kernels
    assert (c_c == c_h).all()
    assert c_h.sum() > 1e8


def test_batched_form_equals_plain_at_full_size(full):
    cl, spec, idx, ctx, qsh = full
    qs = rg.SynthSpec(4321, cl, [120_000, 3_000, 700_000, 50_000], hotspot_fraction=0.1, num_hotspots=8)
    off, sh, rw = rg.synth_batch_layout(qs)
    t = torch.empty((int(off[-1]), 3), dtype=torch.int32, device="cuda:0")
    rg.synth_batch_device(qs, off, t.data_ptr())
    b = rg.DeviceBatch(4, sh, off, t.data_ptr(), rw)
    D = idx.num_sources
    dc = torch.empty((4, D), dtype=torch.int32, device="cuda:0")
    dbp = torch.empty((4, D), dtype=torch.int64, device="cuda:0")
    st = ctx.query_batch_device(b, dc.data_ptr(), dbp.data_ptr(), sub_batch=300_000, graph=True)
    assert st["sub_batches"] > 1
    host = t.cpu().numpy().view(np.uint32)
    bc, bbp = dc.cpu().numpy().view(np.uint32), dbp.cpu().numpy().view(np.uint64)
    for f in range(4):
        per = {}
        for c in range(24):
            a = host[int(off[f * 24 + c]):int(off[f * 24 + c + 1])].copy()
            if len(a):
                a[:, 2] = 0
                per[rg.CHROM_NAMES_24[c]] = a
        pc, pbp, _ = ctx.query_counts(per, 1)
        assert (bc[f] == pc[0]).all() and (bbp[f] == pbp[0]).all(), f


def test_oracle_on_one_full_density_chromosome(full):
    cl, spec, idx, ctx, qsh = full
    c = int(np.argmin(cl))  # the shortest chromosome: ~3.3e7 database intervals
    layers = spec.chrom_layers(c)
    q = qsh[rg.CHROM_NAMES_24[c]]
    oc, _, obp, ost = O.query_database(layers, {c: q.copy()}, 1, idx.num_sources, threads=os.cpu_count() or 1, mode=1)
    gc, gbp, gst = ctx.query_counts({rg.CHROM_NAMES_24[c]: q}, 1)
    assert ost["query_intervals"] == len(q) > 1000
    assert gst["db_swept"] == ost["db_swept"]
    assert (gc == oc).all() and (gbp == obp).all()
    assert oc.sum() > 1e6
