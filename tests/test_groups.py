"""Query length groups (build_query_chrom_data, src/fourier/moments.rs:138-177) against the oracle's
restatement: the host entry point bit for bit, and the device-built groups of a whole batch with
l_int and count exact and the sums within the rounding bound of the reference's sequential sum."""
import numpy as np
import pytest

import oracle as O
import riggle_b200 as rg
from riggle_b200 import api

EPS = np.finfo(np.float64).eps


def lengths_case(rng, kind, n):
    if kind == "random":
        return rng.integers(1, 300_000, n)
    if kind == "bin_multiples":  # every length an exact multiple of the bin: l_int = len / bin exactly
        return 100 * rng.integers(1, 400, n)
    if kind == "short":          # below one bin: l_int = 1
        return rng.integers(1, 100, n)
    if kind == "mixed":
        return np.concatenate([100 * rng.integers(1, 50, n // 3), rng.integers(1, 5000, n - n // 3)])
    raise ValueError(kind)


def intervals(rng, lens, span=200_000_000):
    s = rng.integers(0, span - 300_000, len(lens)).astype(np.uint64)
    return np.stack([s, s + lens.astype(np.uint64), np.zeros(len(lens), np.uint64)], 1).astype(np.uint32)


@pytest.mark.parametrize("kind", ["random", "bin_multiples", "short", "mixed"])
@pytest.mark.parametrize("bin_size", [100, 64])
def test_host_groups_equal_the_oracle(kind, bin_size):
    rng = np.random.default_rng(hash((kind, bin_size)) % 2**32)
    iv = intervals(rng, lengths_case(rng, kind, 5000))
    got = api.query_chrom_groups(iv, bin_size)
    want = O.query_groups(iv[:, 0], iv[:, 1], bin_size)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_host_groups_equal_the_oracle_on_a_million_intervals():
    rng = np.random.default_rng(7)
    iv = intervals(rng, lengths_case(rng, "mixed", 1_000_000))
    got = api.query_chrom_groups(iv)
    want = O.query_groups(iv[:, 0], iv[:, 1])
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def assert_groups_close(got, want, n_bins):
    """got: device groups of one (row, chromosome); want: the oracle's, of which only groups with
    l_int < n_bins are materialised on the device (the store's lookup returns None for the rest)."""
    keep = want[0] < n_bins
    wl, ws, ws2, wc = (w[keep] for w in want)
    gl, gs, gs2, gc = got
    assert np.array_equal(gl, wl) and np.array_equal(gc, wc)
    # the reference adds count terms in sequence (error <= (count - 1) eps of the sum, all terms
    # positive); the device divides one exact integer sum (one rounding)
    tol = (wc.astype(np.float64) + 1) * EPS
    assert np.all(np.abs(gs - ws) <= tol * np.abs(ws))
    assert np.all(np.abs(gs2 - ws2) <= 2 * tol * np.abs(ws2))


@pytest.mark.gpu
def test_device_batch_groups_match_the_oracle():
    import torch

    rng = np.random.default_rng(11)
    cl = np.array([46_709_983, 50_818_468, 20_000_000], np.uint32)
    n_bins = (cl.astype(np.uint64) + 99) // 100
    idx = rg.Index.synth(rg.SynthSpec(3, cl, [2000] * 4))
    ctx = rg.Context(idx)
    mom = api.Moments(4, n_bins)
    kinds = ["random", "bin_multiples", "short", "mixed", "random"]
    sizes = [3000, 2000, 500, 4000, 1_000_000]
    blocks, shards, rows = [], [], []
    for f, (kind, n) in enumerate(zip(kinds, sizes)):
        for c in range(len(cl)):
            if f == 2 and c == 1:
                continue  # a file with no intervals on one chromosome
            lens = lengths_case(rng, kind, n // len(cl))
            if c == 2:
                lens = np.concatenate([lens, [int(n_bins[2]) * 100 + 5]])  # l_int >= n_bins: not materialised
            iv = intervals(rng, lens, span=int(cl[c]))
            iv[:, 2] = f
            blocks.append(iv)
            shards.append(c)
            rows.append(f)
    off = np.zeros(len(blocks) + 1, np.uint64)
    off[1:] = np.cumsum([len(b) for b in blocks])
    allv = np.concatenate(blocks)
    d_iv = torch.from_numpy(allv.view(np.int32)).cuda()
    batch = rg.DeviceBatch(len(kinds), shards, off, d_iv.data_ptr(), rows)
    got = mom.batch_query_groups(ctx, batch, np.arange(len(cl), dtype=np.uint32))
    for f in range(len(kinds)):
        per = dict(got[f])
        for b, (c, r) in enumerate(zip(shards, rows)):
            if r != f:
                continue
            want = O.query_groups(blocks[b][:, 0], blocks[b][:, 1])
            assert_groups_close(per.pop(c), want, int(n_bins[c]))
        assert not per  # no group on a chromosome the file has no intervals on


@pytest.mark.gpu
def test_device_groups_block_local_and_device_wide_forms_agree():
    """With every (file, chromosome) block in ascending order the length keys are sorted within the
    blocks (block-local form); with a file's chromosomes in descending order the batch takes the
    device-wide sort and reduce-by-key.  Both sum exact integers, so the groups must be identical."""
    import torch

    rng = np.random.default_rng(12)
    cl = np.array([46_709_983, 50_818_468, 20_000_000], np.uint32)
    n_bins = (cl.astype(np.uint64) + 99) // 100
    idx = rg.Index.synth(rg.SynthSpec(3, cl, [2000] * 4))
    ctx = rg.Context(idx)
    mom = api.Moments(4, n_bins)
    per_file = {}
    for f, n in enumerate([9000, 300, 60_000]):
        for c in range(len(cl)):
            iv = intervals(rng, lengths_case(rng, "mixed", n), span=int(cl[c]))
            iv[:, 2] = f
            per_file[(f, c)] = iv

    def groups(order):
        blocks = [per_file[k] for k in order]
        off = np.zeros(len(blocks) + 1, np.uint64)
        off[1:] = np.cumsum([len(b) for b in blocks])
        d_iv = torch.from_numpy(np.concatenate(blocks).view(np.int32)).cuda()
        batch = rg.DeviceBatch(3, [k[1] for k in order], off, d_iv.data_ptr(), [k[0] for k in order])
        return mom.batch_query_groups(ctx, batch, np.arange(len(cl), dtype=np.uint32))

    ascending = [(f, c) for f in range(3) for c in range(3)]
    descending = [(f, c) for f in range(3) for c in reversed(range(3))]
    a, d = groups(ascending), groups(descending)
    assert len(a) == len(d) == 3
    for f in range(3):
        ga, gd = dict(a[f]), dict(d[f])
        assert sorted(ga) == sorted(gd)
        for c in ga:
            for x, y in zip(ga[c], gd[c]):
                assert np.array_equal(x, y), (f, c)
