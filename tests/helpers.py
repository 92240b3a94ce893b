"""Shared test data builders (seeded numpy), used with the oracle as the checker."""
import numpy as np

import riggle_b200 as rg


def random_db(rng, n, chrom_len, num_sources, max_len=200_000, edge=True):
    """Random (start, end, sid) intervals with the edge cases the reference's tests exercise:
    touching ends, nested and duplicate starts, sizes at layer-class boundaries."""
    kinds = rng.integers(0, 10, n)
    lens = np.where(kinds < 6, rng.integers(1, 2000, n),
                    np.where(kinds < 8, rng.choice([1, 127, 128, 129, 511, 512, 2047, 2048, 8191, 8192], n),
                             rng.integers(1, max_len, n)))
    lens = np.minimum(lens, chrom_len - 1)
    starts = rng.integers(0, chrom_len - lens, n, dtype=np.int64)
    if edge and n > 10:
        k = n // 10
        starts[:k] = starts[k:2 * k]  # duplicate starts
    ends = starts + lens
    sids = rng.integers(0, num_sources, n)
    return np.stack([starts, ends, sids], 1).astype(np.uint32)


def queries_touching(rng, db, n, rows):
    """Queries that start/end exactly at DB interval ends/starts, plus nested ones."""
    pick = db[rng.integers(0, len(db), n)]
    mode = rng.integers(0, 4, n)
    s = np.where(mode == 0, pick[:, 1], np.where(mode == 1, pick[:, 0] - 50, pick[:, 0] + 1)).astype(np.int64)
    e = np.where(mode == 1, pick[:, 0], np.where(mode == 2, pick[:, 1] - 1, s + rng.integers(1, 5000, n)))
    s = np.maximum(s, 0)
    e = np.maximum(e, s + 1)
    rowsv = rng.integers(0, rows, n)
    return np.stack([s, e, rowsv], 1).astype(np.uint32)


def layers_from_blocks(blocks, cfg=None):
    return rg.bucket_layers(blocks, cfg)
