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
