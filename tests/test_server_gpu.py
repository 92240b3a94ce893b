"""The request server (rgl_server_*): query files submitted one at a time are batched as they arrive
and overlap on the device; every result must be the same alone and in the mix, and equal to the
oracle's.  Needs a GPU."""
import numpy as np
import pytest

import helpers
import oracle as O
import riggle_b200 as rg

pytestmark = pytest.mark.gpu


def _setup(seed, nreq=40, nshards=3, D=17):
    rng = np.random.default_rng(seed)
    blocks = [(sh, helpers.random_db(rng, int(rng.integers(3000, 15000)), 2_000_000, D)) for sh in range(nshards)]
    layers = rg.bucket_layers(blocks)
    reqs = []
    for _ in range(nreq):
        per = {}
        for sh, b in blocks:
            n = int(rng.integers(0, 600))
            if n:
                per[sh] = np.concatenate([helpers.queries_touching(rng, b, n, 1), helpers.random_db(rng, n, 2_000_000, 1)])
        reqs.append(per)
    want = []
    for per in reqs:
        if per:
            c, _, bp, _ = O.query_database(layers, {k: v.copy() for k, v in per.items()}, 1, D)
            want.append((c[0], bp[0]))
        else:
            want.append((np.zeros(D, np.uint32), np.zeros(D, np.uint64)))
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nshards)])
    return idx, reqs, want


def test_alone_equals_mix_equals_oracle():
    idx, reqs, want = _setup(1)
    srv = rg.Server(idx, workers=3)
    alone = []
    for per in reqs:  # one at a time: each request is its own batch
        c, bp, info = srv.wait(srv.submit(per))
        assert info["batch_requests"] == 1
        alone.append((c, bp))
    tickets = [srv.submit(per) for per in reqs]  # all at once: batched as they arrive
    mix = [srv.wait(t) for t in tickets]
    for k in range(len(reqs)):
        assert (alone[k][0] == want[k][0]).all() and (alone[k][1] == want[k][1]).all(), k
        assert (mix[k][0] == want[k][0]).all() and (mix[k][1] == want[k][1]).all(), k
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0 and st["workers"] >= 1
    assert st["p50_ms"] <= st["p99_ms"] <= st["p999_ms"] <= st["max_ms"]
    srv.close()
    idx.close()


def test_single_worker_batches_the_queue():
    idx, reqs, want = _setup(2)
    srv = rg.Server(idx, workers=1, max_batch_requests=64)
    tickets = [srv.submit(per) for per in reqs]
    infos = []
    for k, t in enumerate(tickets):
        c, bp, info = srv.wait(t)
        assert (c == want[k][0]).all() and (bp == want[k][1]).all(), k
        infos.append(info)
    # requests that arrived while the worker was busy ran together
    assert max(i["batch_requests"] for i in infos) > 1
    assert srv.stats()["batches"] < len(reqs)
    srv.close()
    # one query file per launch (the plain path under the same interface)
    srv = rg.Server(idx, workers=1, max_batch_requests=1, counts_only=True)
    tickets = [srv.submit(per, with_overlap=False) for per in reqs]
    for k, t in enumerate(tickets):
        c, bp, info = srv.wait(t)
        assert info["batch_requests"] == 1 and bp is None
        assert (c == want[k][0]).all(), k
    srv.close()
    idx.close()


def test_invalid_request_fails_alone():
    idx, reqs, want = _setup(3, nreq=12)
    srv = rg.Server(idx, workers=1, max_batch_requests=64)
    bad = {0: np.array([[500, 500, 0]], np.uint32)}  # start == end
    tickets = [srv.submit(per) for per in reqs[:6]] + [srv.submit(bad)] + [srv.submit(per) for per in reqs[6:]]
    res = []
    for t in tickets:
        try:
            res.append(srv.wait(t))
        except rg.RiggleError as e:
            res.append(e)
    assert isinstance(res[6], rg.RiggleError)
    good = res[:6] + res[7:]
    for k, r in enumerate(good):
        assert (r[0] == want[k][0]).all() and (r[1] == want[k][1]).all(), k
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == len(reqs)
    # submit-time checks
    with pytest.raises(rg.RiggleError, match="shard id"):
        srv.submit({9: np.array([[1, 5, 0]], np.uint32)})
    srv.close()
    small = rg.Server(idx, workers=1, batch_intervals=100, max_pending_intervals=150)
    with pytest.raises(rg.RiggleError, match="batch_intervals"):
        small.submit({0: np.tile(np.array([[1, 5, 0]], np.uint32), (101, 1))})
    small.close()
    idx.close()


def test_queue_bound_refuses():
    idx, reqs, want = _setup(4, nreq=2)
    srv = rg.Server(idx, workers=1, batch_intervals=1000, max_pending_intervals=50)
    with pytest.raises(rg.RiggleError, match="OOM"):
        srv.submit({0: np.tile(np.array([[1, 5, 0]], np.uint32), (60, 1))})
    srv.close()
    idx.close()


def _moments_for(rng, D, nbins):
    from riggle_b200 import api

    m = api.Moments(D, nbins)
    tables = {}
    for d in range(D):
        for c in range(len(nbins)):
            if rng.random() < 0.15:
                continue
            ns = m.slots(c)
            mean = np.sort(rng.random(ns) * rng.uniform(0.01, 20))
            var = mean * (rng.uniform(1.5, 30) if rng.random() < 0.7 else rng.uniform(0.2, 0.9))
            mv = np.stack([mean, var], 1).astype(np.float32)
            m.set(d, c, mv)
            tables[(d, c)] = mv
    return m, tables


def test_stats_stage_alone_equals_mix_equals_oracle():
    """With a moment store every request also gets its p-values (the stats stage on the device for
    the batch's rows); alone and in the mix they are bit-identical, and equal to the oracle's
    compute_analytic_stats with the oracle's own query length groups (1e-9 relative)."""
    idx, reqs, want = _setup(5, nreq=24)
    D = idx.num_sources
    rng = np.random.default_rng(55)
    nbins = [20_000, 20_000, 20_000]  # the shards span 2 Mbp: 100 bp bins
    m, tables = _moments_for(rng, D, nbins)
    # one worker: the requests submitted while it runs the first one are batched together
    srv = rg.Server(idx, workers=1, max_batch_requests=64, moments=m, shard_chrom=[0, 1, 2])
    alone = [srv.wait(srv.submit(per)) for per in reqs]
    tickets = [srv.submit(per) for per in reqs]
    mix = [srv.wait(t) for t in tickets]
    assert max(r[2]["batch_requests"] for r in mix) > 1  # the mix really ran batched
    checked = 0
    for k, per in enumerate(reqs):
        a, b = alone[k][2]["pvalues"], mix[k][2]["pvalues"]
        for key in ("p", "llr", "lp", "flags"):
            assert np.array_equal(a[key], b[key]), (k, key)
        assert (mix[k][0] == want[k][0]).all() and (mix[k][1] == want[k][1]).all(), k
        groups = [(sh, O.query_groups(v[:, 0], v[:, 1])) for sh, v in sorted(per.items())]
        for d in range(D):
            if not want[k][0][d]:
                assert b["flags"][d] == 0
                continue
            db = {c: (nbins[c], tables[(d, c)]) for c in range(3) if (d, c) in tables}
            w = O.analytic_stats(groups, db, float(want[k][1][d]) / 100.0)
            if w is None:
                assert b["flags"][d] == 0
                continue
            wp, wl = w
            assert b["flags"][d] & 1 and bool(b["flags"][d] & 2) == (wl is not None)
            assert b["p"][d] == pytest.approx(wp, rel=1e-9, abs=1e-300)
            if wl is not None:
                assert b["llr"][d] == pytest.approx(wl, rel=1e-9, abs=1e-12)
            checked += 1
    assert checked > 50
    srv.close()
    m.close()
    idx.close()


def test_admission_by_free_device_memory():
    """Admission happens when a batch is formed, against the free device memory the server sees
    (here a provider injected from the host): with none free, only requests that fit the workers'
    initial workspaces run and the rest fail with RGL_ERR_OOM; once memory is reported free again,
    the same large request is admitted (its worker's workspace grows) and is exact."""
    idx, reqs, want = _setup(6, nreq=6)
    free = {"bytes": 0}
    srv = rg.Server(idx, workers=2, initial_intervals=1000, hbm_reserve_bytes=1 << 20,
                    free_memory=lambda: free["bytes"])
    small = {0: reqs[0][0][:200]} if 0 in reqs[0] else {1: reqs[0][1][:200]}
    big = {sh: np.tile(v, (8, 1)) for sh, v in reqs[1].items()}
    assert sum(len(v) for v in big.values()) > 1000
    c, bp, info = srv.wait(srv.submit(small))
    layers = {k: idx.export_layer(*k) for k in [(s_, l) for s_ in range(3) for l in range(idx.num_layer_slots)
                                                if idx.layer_count(s_, l)]}
    wc, _, wbp, _ = O.query_database(layers, {k: v.copy() for k, v in small.items()}, 1, idx.num_sources)
    assert (c == wc[0]).all() and (bp == wbp[0]).all()
    with pytest.raises(rg.RiggleError) as e:
        srv.wait(srv.submit(big))
    assert e.value.status == rg._lib.RGL_ERR_OOM
    st = srv.stats()
    assert st["refused"] == 1 and st["grown_bytes"] == 0
    free["bytes"] = 1 << 50  # memory frees up: the next formation admits it
    c, bp, info = srv.wait(srv.submit(big))
    wc, _, wbp, _ = O.query_database(layers, {k: v.copy() for k, v in big.items()}, 1, idx.num_sources)
    assert (c == wc[0]).all() and (bp == wbp[0]).all()
    assert srv.stats()["grown_bytes"] > 0
    srv.close()
    idx.close()
