"""Results on the way out: the non-zero cells as CSR (K9, on the device) and the reference's JSON
output (src/main.rs:141-204, src/stats/mod.rs), against the oracle's restatements."""
import numpy as np
import pytest

import oracle as O
from riggle_b200 import api

PV_EMITTED, PV_HAS_LLR = 1, 2


@pytest.mark.parametrize("v", [0.0, -0.0, 1.0, 420.0, 1e-5, 1e-6, 12.3, 0.5, 1e15, 1e16, 1e17, 123456789.0,
                               1.2345678901234568e17, 1e-300, 5e-324, 1.7976931348623157e308, 0.1572992,
                               3.0e-5, 2.5e-7, 99999999999999.9, 0.30000000000000004, float("inf"), float("nan")])
def test_float_layout_matches_serde(v):
    got = api.stats_json([0, 1], [0], [1], ["q"], ["d"], 1, observed_bins=[v], p_value=[0.5], llr=[0.0],
                         flags=[PV_EMITTED])
    assert f'"observed_bins": {O.json_f64(v)},' in got


def test_known_float_strings():
    # serde_json's layout for a few values (plain decimal, integers with ".0", exponents without '+')
    for v, s in [(1e-5, "0.00001"), (420.0, "420.0"), (1e16, "1e16"), (1e15, "1000000000000000.0"),
                 (1e-300, "1e-300"), (2.5e-7, "2.5e-7"), (12.3, "12.3"), (1.2345678901234568e17, "1.2345678901234568e17")]:
        assert O.json_f64(v) == s


def test_reference_json_known_answers():
    """src/stats/mod.rs:66-100: without stats no p_value / llr keys; with stats all three keys."""
    plain = api.stats_json([0, 1], [0], [42], ["q.bed"], ["db.bed"], 1)
    assert "overlap_count" in plain and "p_value" not in plain and "llr" not in plain
    assert plain == O.json_pretty("results", [[("query_name", "q.bed"), ("db_name", "db.bed"), ("overlap_count", 42)]])
    stats = api.stats_json([0, 1], [0], [42], ["q.bed"], ["db.bed"], 1, observed_bins=[420.0], p_value=[1e-5],
                           llr=[12.3], flags=[PV_EMITTED | PV_HAS_LLR])
    assert "p_value" in stats and "observed_bins" in stats and "llr" in stats
    assert stats == ('{\n  "results": [\n    {\n      "query_name": "q.bed",\n      "db_name": "db.bed",\n'
                     '      "overlap_count": 42,\n      "observed_bins": 420.0,\n      "p_value": 0.00001,\n'
                     '      "llr": 12.3\n    }\n  ]\n}')
    assert api.stats_json([0], [], [], [], ["db.bed"], 1) == '{\n  "results": []\n}'


def _oracle_stats_json(counts, qn, dn, obs=None, p=None, llr=None, flags=None):
    """main.rs:141-204 restated: entries from the CSR (stats: emitted cells only), sorted."""
    indptr, indices, data = O.dense_to_csr(counts)
    es = []
    for q in range(counts.shape[0]):
        for e in range(int(indptr[q]), int(indptr[q + 1])):
            d = int(indices[e])
            if p is not None and not flags[q, d] & PV_EMITTED:
                continue
            es.append((q, d, int(data[e])))
    if p is not None:
        es.sort(key=lambda t: p[t[0], t[1]])  # stable: ties in (query, database) order
    else:
        es.sort(key=lambda t: -t[2])
    objs = []
    for q, d, c in es:
        o = [("query_name", qn[q]), ("db_name", dn[d]), ("overlap_count", c)]
        if p is not None:
            o += [("observed_bins", float(obs[q, d])), ("p_value", float(p[q, d]))]
            if flags[q, d] & PV_HAS_LLR:
                o.append(("llr", float(llr[q, d])))
        objs.append(o)
    return O.json_pretty("results", objs)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_stats_json_matches_the_restated_writer(seed):
    rng = np.random.default_rng(seed)
    R, D = 7, 11
    counts = (rng.integers(0, 4, (R, D)) * (rng.random((R, D)) < 0.5)).astype(np.uint32)
    counts[2] = 0
    qn = [f"q{i}.bed" for i in range(R)]
    dn = [f'db "{i}"\t.bed' for i in range(D)]  # escaped characters in names
    indptr, indices, data = O.dense_to_csr(counts)
    assert api.stats_json(indptr, indices, data, qn, dn, D) == _oracle_stats_json(counts, qn, dn)
    p = rng.choice([1e-300, 1e-7, 0.25, 1.0, 0.0312], (R, D))
    obs = rng.random((R, D)) * 1e3
    llr = rng.random((R, D)) * 50
    flags = np.where(counts > 0, PV_EMITTED | (rng.random((R, D)) < 0.7) * PV_HAS_LLR, 0).astype(np.uint8)
    flags[0, :] &= ~np.uint8(PV_EMITTED)  # a row without shared chromosomes: nothing emitted
    got = api.stats_json(indptr, indices, data, qn, dn, D, obs, p, llr, flags)
    assert got == _oracle_stats_json(counts, qn, dn, obs, p, llr, flags)


def test_intervals_json():
    pairs = np.array([[10, 20, 15, 30, 1, 0, 2, 5], [0, 5, 1, 2, 0, 1, 0, 1]], np.uint32)
    got = api.intervals_json(pairs, ["a.bed", "b.bed"], ["x.bed", "y.bed"], ["chr1", "chr2", "chr3"])
    want = O.json_pretty("hits", [
        [("query_name", "b.bed"), ("db_name", "x.bed"), ("chrom", "chr3"), ("query_start", 10), ("query_end", 20),
         ("db_start", 15), ("db_end", 30), ("intersection_bp", 5)],
        [("query_name", "a.bed"), ("db_name", "y.bed"), ("chrom", "chr1"), ("query_start", 0), ("query_end", 5),
         ("db_start", 1), ("db_end", 2), ("intersection_bp", 1)]])
    assert got == want
    assert api.intervals_json(np.zeros((0, 8), np.uint32), ["a"], ["x"], ["c"]) == '{\n  "hits": []\n}'


@pytest.mark.gpu
@pytest.mark.parametrize("R,D,density", [(1, 1, 1.0), (5, 31, 0.3), (64, 1000, 0.05), (300, 33, 0.0),
                                         (4096, 1000, 0.2), (3, 70, 1.0)])
def test_dense_to_csr_on_the_device(R, D, density):
    import torch

    import riggle_b200 as rg

    rng = np.random.default_rng(R * 7 + D)
    counts = (rng.integers(1, 2**32, (R, D), dtype=np.uint64) * (rng.random((R, D)) < density)).astype(np.uint32)
    if R > 3:
        counts[R // 2] = 0  # an empty row
    bp = rng.integers(0, 2**63, (R, D), dtype=np.uint64)
    idx = rg.Index.synth(rg.SynthSpec(3, np.array([2_000_000], np.uint32), [100]))
    ctx = rg.Context(idx)
    dc = torch.from_numpy(counts.view(np.int32)).cuda()
    db = torch.from_numpy(bp.view(np.int64)).cuda()
    indptr, ind, val, bpv = api.dense_to_csr_device(ctx, dc.data_ptr(), R, D, db.data_ptr())
    wi, wind, wval = O.dense_to_csr(counts)
    assert np.array_equal(indptr, wi) and np.array_equal(ind, wind) and np.array_equal(val, wval)
    rows = np.repeat(np.arange(R), np.diff(wi.astype(np.int64)))
    assert np.array_equal(bpv, bp[rows, wind])
