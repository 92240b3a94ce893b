"""FP64 p-values on the GPU (through the C ABI) against the oracle's restatement of
compute_analytic_stats.  Needs a GPU."""
import numpy as np
import pytest

import oracle as O
import riggle_b200 as rg
from riggle_b200 import api

pytestmark = pytest.mark.gpu

NB = {"chr21": (46_709_983 + 99) // 100, "chr22": (50_818_468 + 99) // 100}


def oracle_cell(row_groups, tables, d, observed):
    """tables: {(sid, chrom): mv}; n_bins per chrom from `nbins`."""
    db = {c: (nb, tables[(d, c)]) for c, nb in enumerate(nbins) if (d, c) in tables}
    return O.analytic_stats([(c, g) for c, g in row_groups], db, observed)


nbins = [NB["chr21"], NB["chr22"], 2000, 5]


def random_case(rng, rows, D):
    m = api.Moments(D, nbins)
    tables = {}
    for d in range(D):
        for c in range(len(nbins)):
            if rng.random() < 0.2:
                continue  # source has no intervals on this chromosome
            ns = m.slots(c)
            mean = np.sort(rng.random(ns) * rng.uniform(0.01, 50))
            kind = rng.integers(0, 3)
            var = mean * (rng.uniform(1.5, 30) if kind else rng.uniform(0.1, 0.9))  # over / under-dispersed
            mv = np.stack([mean, var], 1).astype(np.float32)
            if rng.random() < 0.1:
                mv = mv[: ns // 2]  # a shorter table: lookups past it return None
            m.set(d, c, mv)
            tables[(d, c)] = mv
    row_groups, oracle_groups = [], []
    for q in range(rows):
        chroms, ochroms = [], []
        for c in range(len(nbins)):
            if rng.random() < 0.3:
                continue
            n = int(rng.integers(1, 400))
            lens = np.concatenate([rng.integers(1, 3000, n), rng.integers(1, 300_000, 5)])
            ivs = np.stack([np.zeros(len(lens)), lens, np.zeros(len(lens))], 1).astype(np.uint32)
            chroms.append((c, api.query_chrom_groups(ivs)))
            ochroms.append((c, O.query_groups(ivs[:, 0], ivs[:, 1])))
        row_groups.append(chroms)
        oracle_groups.append(ochroms)
    counts = rng.integers(0, 3, (rows, D)).astype(np.uint32)
    bp = (rng.random((rows, D)) * rng.choice([10, 1e4, 1e7], (rows, D))).astype(np.uint64)
    return m, tables, row_groups, oracle_groups, counts, bp


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_pvalues_match_oracle(seed):
    rng = np.random.default_rng(seed)
    rows, D = 9, 13
    m, tables, row_groups, oracle_groups, counts, bp = random_case(rng, rows, D)
    p, llr, lp, fl = m.pvalues(row_groups, counts, bp)
    n_emit = 0
    for q in range(rows):
        for d in range(D):
            want = None
            if counts[q, d]:
                want = oracle_cell(oracle_groups[q], tables, d, float(bp[q, d]) / 100.0)
            if want is None:
                assert fl[q, d] == 0 and p[q, d] == 1.0
                continue
            n_emit += 1
            wp, wl = want
            assert fl[q, d] & 1
            assert bool(fl[q, d] & 2) == (wl is not None)
            if wl is not None:
                assert llr[q, d] == pytest.approx(wl, rel=1e-9, abs=1e-12)
            if wp > 1e-290:
                assert p[q, d] == pytest.approx(wp, rel=1e-9)
            if p[q, d] > 1e-290:
                assert lp[q, d] == pytest.approx(np.log(p[q, d]), rel=1e-9, abs=1e-12)
    assert n_emit > 20


def test_reference_stats_known_answers():
    """src/fourier/stats.rs:195-214 with moments fixed at (20, 100), through the device path."""
    m = api.Moments(1, [NB["chr22"]])
    m.set(0, 0, np.tile(np.array([20.0, 100.0], np.float32), (m.slots(0), 1)))
    g = api.query_chrom_groups(np.array([[0, 1000, 0]], np.uint32))
    p, llr, lp, fl = m.pvalues([[(0, g)]], np.array([[1]], np.uint32), np.array([[0]], np.uint64))
    assert p[0, 0] == 1.0  # observed 0: NB p_o = 1 fails the bounds -> p = 1
    p, llr, lp, fl = m.pvalues([[(0, g)]], np.array([[1]], np.uint32), np.array([[1000]], np.uint64))
    assert 0.5 < p[0, 0] < 1.0  # observed 10 bins < mu 20: depleted
    # zero count: not emitted (src/tasks/query/pvalues.rs:28-35)
    p, llr, lp, fl = m.pvalues([[(0, g)]], np.array([[0]], np.uint32), np.array([[1000]], np.uint64))
    assert fl[0, 0] == 0


def test_deep_tail_in_log_space():
    m = api.Moments(1, [NB["chr22"]])
    m.set(0, 0, np.tile(np.array([2.0, 8.0], np.float32), (m.slots(0), 1)))
    g = api.query_chrom_groups(np.array([[0, 1000, 0]] * 50, np.uint32))
    # a huge observation: p underflows to 0 in linear space, ln p stays finite
    p, llr, lp, fl = m.pvalues([[(0, g)]], np.array([[1]], np.uint32), np.array([[10**9]], np.uint64))
    assert p[0, 0] == 0.0 and np.isfinite(lp[0, 0]) and lp[0, 0] < -700
    want = O.lib().orc_log_p(llr[0, 0], 1, 1e7, 100.0)
    assert lp[0, 0] == pytest.approx(want, rel=1e-12)


def test_end_to_end_counts_moments_pvalues():
    """Sweep counts on the GPU, moments from the oracle's restatement of the reference's FFT
    pipeline, p-values on the GPU vs the oracle: two hg38 chromosomes, 6 DB files, 2 query files."""
    cl = np.array([46_709_983, 50_818_468], np.uint32)  # chr21, chr22 of the hg38 table
    dbs = rg.SynthSpec(5, cl, [4000] * 6, broad_fraction=0.02)
    qs = rg.SynthSpec(77, cl, [800, 3000])
    idx = rg.Index.synth(dbs)
    ctx = rg.Context(idx)
    shards = {}
    for c in range(2):
        blocks = []
        for f in range(2):
            b = qs.block(f, c).copy()
            b[:, 2] = f
            blocks.append(b)
        shards[idx.shard_name(c)] = np.concatenate(blocks)
    counts, bp, _ = ctx.query_counts(shards, 2)
    m = api.Moments(6, [NB["chr21"], NB["chr22"]])
    tables = {}
    for f in range(6):
        for c in range(2):
            iv = dbs.block(f, c)
            g = O.depth_signal(iv[:, 0], iv[:, 1], nbins[c])
            mv, _, _ = O.moments_from_signal(g)
            m.set(f, c, mv)
            tables[(f, c)] = mv
    row_groups = [[(c, api.query_chrom_groups(qs.block(f, c))) for c in range(2)] for f in range(2)]
    oracle_groups = [[(c, O.query_groups(qs.block(f, c)[:, 0], qs.block(f, c)[:, 1])) for c in range(2)]
                     for f in range(2)]
    p, llr, lp, fl = m.pvalues(row_groups, counts, bp)
    for q in range(2):
        for d in range(6):
            if not counts[q, d]:
                continue
            wp, wl = oracle_cell(oracle_groups[q], tables, d, float(bp[q, d]) / 100.0)
            assert p[q, d] == pytest.approx(wp, rel=1e-9, abs=1e-300)
            if wl is not None:
                assert llr[q, d] == pytest.approx(wl, rel=1e-9)
