"""Sliding-window moments on the GPU (K4-K7) against the oracle.  Needs a GPU.

The depth signal must match the reference's f32 signal bit for bit; the moments are compared with
the oracle's exact (double-double, direct) window moments of that signal.  The reference's own
d*-autocorrelation formula (the oracle's restatement of moments_from_signal) is reported beside it:
its cancellation leaves it far less accurate than the device's centred formulation."""
import numpy as np
import pytest

import oracle as O
import riggle_b200 as rg
from riggle_b200 import api

pytestmark = pytest.mark.gpu


def rand_intervals(rng, n, span, maxlen=5000):
    s = rng.integers(0, span, n).astype(np.int64)
    e = s + rng.integers(1, maxlen, n)
    # exact bin boundaries, shared bins, intervals past the chromosome end (clipped)
    s[: n // 10] = (s[: n // 10] // 100) * 100
    e[n // 10: n // 5] = (e[n // 10: n // 5] // 100 + 1) * 100
    e[-3:] = span + 5000
    iv = np.stack([s, e, np.zeros(n)], 1).astype(np.uint32)
    return iv


@pytest.mark.parametrize("n_bins,n", [(7, 3), (8, 5), (1000, 200), (20_001, 3000), (65_536, 20_000)])
def test_depth_signal_bit_exact(n_bins, n):
    rng = np.random.default_rng(n_bins)
    iv = rand_intervals(rng, n, n_bins * 100)
    g = api.depth_signal(iv, n_bins)
    want = O.depth_signal(iv[:, 0], iv[:, 1], n_bins)
    assert np.array_equal(g, want) or np.array_equal(g.view(np.uint32) & 0x7FFFFFFF, want.view(np.uint32) & 0x7FFFFFFF)
    assert (g == want).all()


def test_depth_signal_empty_and_tiny():
    assert (api.depth_signal(np.zeros((0, 3), np.uint32), 10) == 0).all()
    g = api.depth_signal(np.array([[20, 80, 0]], np.uint32), 1)
    assert (g == O.depth_signal(np.array([20], np.uint32), np.array([80], np.uint32), 1)).all()


def build(intervals, n_bins):
    m = api.Moments(1, [n_bins])
    mean, var = m.build(0, 0, intervals, report=True)
    return m, mean, var


@pytest.mark.parametrize("seed,n_bins,n", [(1, 30_000, 400), (2, 50_000, 3000), (3, 40_000, 20)])
def test_moments_match_exact_oracle(seed, n_bins, n):
    rng = np.random.default_rng(seed)
    iv = rand_intervals(rng, n, n_bins * 100, maxlen=20_000)
    m, mean, var = build(iv, n_bins)
    g = O.depth_signal(iv[:, 0], iv[:, 1], n_bins)
    grid = O.moment_grid(n_bins)
    em, ev = O.moments_exact(g, grid, threads=8)
    _, rm, rv = O.moments_from_signal(g)  # the reference's formula, FP64
    scale = np.maximum(np.abs(ev), 1e-12 * em * em + 1e-300)
    err_gpu_var = np.max(np.abs(var - ev) / scale)
    err_gpu_mean = np.max(np.abs(mean - em) / np.maximum(np.abs(em), 1e-300))
    err_ref_var = np.max(np.abs(rv - ev) / scale)
    print(f"n_bins={n_bins}: device var rel err {err_gpu_var:.2e}, mean {err_gpu_mean:.2e}; "
          f"reference formula var rel err {err_ref_var:.2e}")
    assert err_gpu_mean < 1e-9
    assert err_gpu_var < 1e-6
    # the stored f32 pairs are the FP64 values rounded
    stored = m.get(0, 0)
    assert np.array_equal(stored[:, 0], mean.astype(np.float32))
    assert np.array_equal(stored[:, 1], var.astype(np.float32))


def test_reference_window_moment_known_answers():
    # uniform coverage: mean(L) = L, var(L) = 0 (src/fourier/moments.rs:511-538)
    m, mean, var = build(np.array([[0, 5000, 0]], np.uint32), 50)
    grid = O.moment_grid(50)
    np.testing.assert_allclose(mean, grid, atol=1e-9)
    assert np.all(var < 1e-9)
    # g = [1,0,0,1,0,0,1]: L = 3 -> mean 1, var 0; mean(L=1) = 3/7 (src/fourier/moments.rs:540-562)
    iv = np.array([[0, 100, 0], [300, 400, 0], [600, 700, 0]], np.uint32)
    m, mean, var = build(iv, 7)
    assert abs(mean[2] - 1.0) < 1e-12 and var[2] < 1e-12
    assert abs(mean[0] - 3.0 / 7.0) < 1e-12


def test_chr22_lookups_like_the_reference():
    # src/fourier/moments.rs:566-592 on chr22 of the hg38 table
    nb = (50_818_468 + 99) // 100
    m, mean, var = build(np.array([[10_000_000, 20_000_000, 0]], np.uint32), nb)
    i = rg.api.compact_index(50)
    assert mean[i] > 0 and var[i] >= 0
    m, mean, var = build(np.array([[0, 50_818_468, 0]], np.uint32), nb)
    i = rg.api.compact_index(500)
    assert abs(mean[i] - 500) / 500 < 0.02


def test_moments_feed_pvalues_like_the_reference_integration_test():
    """Self query most enriched (tests/integration.rs:119-181, with seeded synthetic files of this
    build's generator): p(self) < p(other) and p(self) < 1e-10."""
    cl = np.array([46_709_983, 50_818_468], np.uint32)
    nbins = [(int(x) + 99) // 100 for x in cl]
    files = rg.SynthSpec(77, cl, [2000, 2000])
    idx = rg.Index.synth(files)
    m = api.Moments(2, nbins)
    for f in range(2):
        for c in range(2):
            m.build(f, c, files.block(f, c))
    ctx = rg.Context(idx)
    q = {idx.shard_name(c): files.block(0, c) * np.array([1, 1, 0], np.uint32) for c in range(2)}
    counts, bp, _ = ctx.query_counts(q, 1)
    groups = [[(c, api.query_chrom_groups(files.block(0, c))) for c in range(2)]]
    p, llr, lp, fl = m.pvalues(groups, counts, bp)
    assert fl[0, 0] & 1 and fl[0, 1] & 1
    assert p[0, 0] < p[0, 1] and p[0, 0] < 1e-10


def _grid_subset(n_bins, stride):
    """Grid indices with L in [2^8, 2^16] (every `stride`-th) plus the grid's first, last and a few
    L below 2^8, so that every size class of window is covered."""
    grid = O.moment_grid(n_bins)
    mid = np.nonzero((grid >= 256) & (grid <= 65_536))[0][::stride]
    edge = np.array([0, 1, 50, 99, 150, len(grid) - 1])
    return grid, np.unique(np.concatenate([mid, edge[edge < len(grid)]]))


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("n_bins,bin_size,n,stride", [
    (1 << 20, 100, 60_000, 1),      # every grid L
    (1 << 20, 64, 60_000, 1),
    (1 << 22, 64, 200_000, 3),
    (1 << 22, 100, 200_000, 3),
    (1 << 23, 64, 300_000, 6),
    (1 << 21, 64, 2_000, 3),        # sparse: the last windows' variance is ~1e-10 of their mean^2
])
def test_moments_at_precision_sizes(n_bins, bin_size, n, stride, precision):
    """Config-3 sizes (2^20-2^23 bins, 64 and 100 bp bins, FFT lengths up to 2^25): the device's
    moments, FP64 or compensated FP32 (FP64 only in the final reduction), against the oracle's exact
    (double-double, direct) window moments, for L in [2^8, 2^16] and the grid's edges.  Variance
    within 1e-6 relative in both; mean within 1e-9 (FP64) or 1e-6 (compensated FP32)."""
    rng = np.random.default_rng(n_bins + bin_size)
    span = n_bins * bin_size
    spec = rg.SynthSpec(int(rng.integers(1, 1 << 30)), np.array([min(span, 2**32 - 1)], np.uint32), [n],
                        broad_fraction=0.05)
    iv = spec.block(0, 0)
    m = api.Moments(1, [n_bins])
    mean, var = m.build(0, 0, iv, bin_size=bin_size, report=True, precision=precision)
    g = O.depth_signal(iv[:, 0], iv[:, 1], n_bins, bin_size)
    grid, sel = _grid_subset(n_bins, stride)
    em, ev = O.moments_exact(g, grid[sel], threads=0)
    scale = np.maximum(np.abs(ev), 1e-12 * em * em + 1e-300)
    err_var = np.abs(var[sel] - ev) / scale
    err_mean = np.abs(mean[sel] - em) / np.maximum(np.abs(em), 1e-300)
    mid = (grid[sel] >= 256) & (grid[sel] <= 65_536)
    print(f"{precision} n_bins=2^{int(np.log2(n_bins))} bin={bin_size}: {len(sel)} L; max rel err mean "
          f"{err_mean.max():.2e}, var {err_var.max():.2e} (L in [2^8, 2^16]: mean {err_mean[mid].max():.2e}, "
          f"var {err_var[mid].max():.2e})")
    assert err_mean.max() < (1e-9 if precision == "fp64" else 1e-6)
    assert err_var.max() < 1e-6
