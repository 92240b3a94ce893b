"""`--intervals` mode on the GPU (rgl_query_pairs) against the oracle's restatement of
query_sweep_pairs / collect_interval_pairs.  Needs a GPU."""
import numpy as np
import pytest

import helpers
import oracle as O
import riggle_b200 as rg

pytestmark = pytest.mark.gpu


def _sorted(a):
    return a[np.lexsort(a.T[::-1])]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_pairs_equal_oracle_and_counts(seed):
    rng = np.random.default_rng(seed)
    rows, D, nsh = int(rng.integers(1, 9)), int(rng.integers(1, 20)), 3
    blocks = [(sh, helpers.random_db(rng, int(rng.integers(100, 15000)), 3_000_000, D)) for sh in range(nsh)]
    layers = rg.bucket_layers(blocks)
    qsh = {sh: np.concatenate([helpers.queries_touching(rng, b, 400, rows), helpers.random_db(rng, 400, 3_000_000, rows)])
           for sh, b in blocks}
    want = O.query_pairs(layers, {k: v.copy() for k, v in qsh.items()})
    idx = rg.Index.from_layers(layers, D, [f"s{i}" for i in range(nsh)])
    ctx = rg.Context(idx)
    got = ctx.query_pairs(qsh, rows)
    assert got.shape == want.shape and len(got) > 100
    assert (_sorted(got) == _sorted(want)).all()
    # the device order is (layer, shard, row, query start, db start): deterministic across calls
    assert (ctx.query_pairs(qsh, rows) == got).all()
    # the structural invariants of the reference's own intervals test (tests/integration.rs:78-101)
    assert (got[:, 0] < got[:, 1]).all() and (got[:, 2] < got[:, 3]).all() and (got[:, 7] > 0).all()
    assert (np.minimum(got[:, 1], got[:, 3]) - np.maximum(got[:, 0], got[:, 2]) == got[:, 7]).all()
    # pairs aggregate to the count / overlap matrix
    c, bp, _ = ctx.query_counts(qsh, rows)
    cc = np.zeros((rows, D), np.uint64)
    np.add.at(cc, (got[:, 4], got[:, 5]), 1)
    bb = np.zeros((rows, D), np.uint64)
    np.add.at(bb, (got[:, 4], got[:, 5]), got[:, 7].astype(np.uint64))
    assert (cc == c).all() and (bb == bp).all()
    ctx.close()
    idx.close()


def test_pairs_capacity_and_empty():
    rng = np.random.default_rng(5)
    db = helpers.random_db(rng, 4000, 500_000, 4)
    layers = rg.bucket_layers([(0, db)])
    idx = rg.Index.from_layers(layers, 4, ["s0"])
    ctx = rg.Context(idx)
    assert ctx.query_pairs({}, 1).shape == (0, 8)
    far = np.array([[900_000, 900_100, 0]], np.uint32)  # beyond every DB interval
    assert ctx.query_pairs({0: far}, 1).shape == (0, 8)
    q = helpers.queries_touching(rng, db, 200, 1)
    full = ctx.query_pairs({0: q}, 1)
    import ctypes as C

    from riggle_b200 import _lib

    keep = []
    batch = ctx._batch({0: q}, 1, keep)
    out = np.empty((len(full) - 1, 8), np.uint32)
    n = C.c_uint64()
    st = _lib.load().rgl_query_pairs(ctx._h, C.byref(batch), len(full) - 1, out.ctypes.data_as(C.c_void_p),
                                     C.byref(n))
    assert st == _lib.RGL_ERR_INVALID_ARGUMENT and n.value == len(full)
    bad = q.copy()
    bad[0, 1] = bad[0, 0]
    with pytest.raises(rg.RiggleError, match="INVALID_ARGUMENT"):
        ctx.query_pairs({0: bad}, 1)
    assert (ctx.query_pairs({0: q}, 1) == full).all()
    ctx.close()
    idx.close()
