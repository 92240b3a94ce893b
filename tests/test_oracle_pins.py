"""Pins the CPU oracle to the reference's own known answers (tests/golden/known_answers.json,
transcribed from the reference crate's unit tests).  CPU only."""
import numpy as np
import pytest

import oracle as O


def test_sweep_known_answers(known):
    for case in known["sweep"]:
        counts, bins = O.query_sweep(case["db"], case["layer_max"], case["query"], case["rows"], case["cols"])
        assert counts.tolist() == case["counts"], case["ref"]
        np.testing.assert_allclose(bins, np.array(case["bins"], np.float32), atol=1e-5, err_msg=case["ref"])


def test_layer_config_known_answers(known):
    lf = known["layer_for_size"]
    for size, k in lf["cases"]:
        assert O.lib().orc_layer_for_size(lf["min_size"], lf["growth_factor"], size) == k
    lm = known["layer_max_size"]
    for layer, mx in lm["cases"]:
        assert O.lib().orc_layer_max_size(lm["min_size"], lm["growth_factor"], layer) == mx
    # tile_size = layer_max_size / 2, minimum 1 (src/io/meta.rs:79-81)
    assert O.lib().orc_tile_size(128, 4, 0) == 64
    assert O.lib().orc_tile_size(1, 2, 0) == 1


def test_layer_config_general_path():
    # non-power-of-two config takes the threshold loop (src/io/meta.rs:49-57)
    L = O.lib()
    for size in [0, 99, 100, 299, 300, 899, 900, 2699, 2700, 10**9]:
        k, thr = 0, 100
        while thr <= size:
            thr *= 3
            k += 1
        assert L.orc_layer_for_size(100, 3, size) == k


def test_jump_table_known_answers(known):
    for c in known["jump_build"]:
        assert O.build_jump_table(c["starts"], c["tile"]).tolist() == c["table"], c["ref"]
    for c in known["jump_lookup"]:
        for target, want in c["cases"]:
            assert O.jump_lookup(c["table"], c["tile"], target) == want, c["ref"]
    for c in known["jump_extend"]:
        t = O.extend_jump_table(c["old"], c["new_starts"], c["tile"])
        for target, want in c["lookups"]:
            assert O.jump_lookup(t, c["tile"], target) == want, c["ref"]


def test_jump_table_matches_partition_point_random():
    rng = np.random.default_rng(5)
    for _ in range(20):
        starts = np.sort(rng.integers(0, 100000, rng.integers(1, 500))).astype(np.uint32)
        tile = int(rng.integers(1, 3000))
        t = O.build_jump_table(starts, tile)
        for i, v in enumerate(t):
            assert v == np.searchsorted(starts, i * tile, side="left")


def test_layer_extend_known_answers(known):
    for c in known["layer_extend"]:
        old = np.array(c["old"], np.uint32).reshape(-1, 3)
        pos, sid = O.extend_layer(old[:, :2], old[:, 2], c["new"])
        assert pos[:, 0].tolist() == c["starts"], c["ref"]
        if "sids" in c:
            assert sid.tolist() == c["sids"], c["ref"]


def test_depth_total_cov(known):
    c = known["depth_total_cov"]
    n_bins = (50_818_468 + 99) // 100  # chr22 in the hg38 table (src/fourier/genome.rs:28)
    iv = np.array(c["intervals"], np.uint32)
    g = O.depth_signal(iv[:, 0], iv[:, 1], n_bins)
    assert abs(float(np.sum(g, dtype=np.float64)) - c["total_cov"]) < c["tol"] * 10


def test_cumsum_known_answers():
    # src/fourier/depth.rs:232-268
    x = (np.arange(100) * 0.5 - 25.0).astype(np.float32)
    np.testing.assert_allclose(O.cumsum_f32(x), np.cumsum(x.astype(np.float64)), atol=1e-4)
    y = np.arange(1, 12, dtype=np.float32)
    np.testing.assert_allclose(O.cumsum_f32(y), np.cumsum(y), atol=1e-4)


def test_autocorr_known_answers(known):
    for c in known["autocorr"]:
        r = O.autocorr(c["x"])
        assert abs(r[c["lag"]] - c["value"]) < c["tol"], c["ref"]


def test_autocorr_matches_numpy():
    rng = np.random.default_rng(1)
    x = rng.random(1000) * 100
    r = O.autocorr(x)
    ref = np.correlate(x, x, mode="full")[len(x) - 1:]
    np.testing.assert_allclose(r, ref, rtol=1e-9, atol=1e-6)


def test_d2_prefix_sum():
    # src/fourier/moments.rs:492-507
    x = np.arange(20) * 0.7
    got = O.d2_prefix_sum(x)
    want = np.concatenate([[0.0], np.cumsum(x * x)])
    np.testing.assert_allclose(got, want, atol=1e-9)


def test_window_moments_known_answers(known):
    for l in range(1, 50):  # moments.rs:511-538, uniform signal of 50 ones
        m, v = O.window_moments_from_g(np.ones(50, np.float32), l)
        assert abs(m - l) < 1e-6 and v < 1e-6
    c = known["window_moments"][1]
    for l, mean, var in c["cases"]:
        m, v = O.window_moments_from_g(c["g"], l)
        assert abs(m - mean) < 1e-6
        if var is not None:
            assert v < 1e-6


def test_chrom_moments_lookups():
    # src/fourier/moments.rs:566-602 on chr22 (n_bins 508185)
    n_bins = (50_818_468 + 99) // 100
    def lookup(mv, l):
        l = int(np.ceil(l))
        if l == 0 or l >= n_bins:
            return None
        i = O.compact_index(l)
        return None if i >= len(mv) else (float(mv[i, 0]), float(mv[i, 1]))
    g = O.depth_signal(np.array([10_000_000], np.uint32), np.array([20_000_000], np.uint32), n_bins)
    mv, _, _ = O.moments_from_signal(g)
    r = lookup(mv, 50.0)
    assert r is not None and r[0] > 0 and r[1] >= 0
    g = O.depth_signal(np.array([0], np.uint32), np.array([50_818_468], np.uint32), n_bins)
    mv, _, _ = O.moments_from_signal(g)
    m, _ = lookup(mv, 500.0)
    assert abs(m - 500) / 500 < 0.02
    g = O.depth_signal(np.array([0], np.uint32), np.array([1_000_000], np.uint32), n_bins)
    mv, _, _ = O.moments_from_signal(g)
    assert lookup(mv, 0.0) is None and lookup(mv, float(n_bins)) is None


def test_compact_index_and_grid():
    # moments.rs:58-66 and 215-247: dense below 101, then one slot per log_1.01 step
    assert [O.compact_index(l) for l in (1, 50, 100)] == [0, 49, 99]
    assert O.compact_index(101) == 100
    grid = O.moment_grid(508185)
    assert grid[:100].tolist() == list(range(1, 101))
    assert all(b > a for a, b in zip(grid[:-1], grid[1:]))
    # ~T + log_1.01(N/T) entries (docs/stats.md: ~1100 for chr1, fewer for chr22)
    assert abs(len(grid) - (100 + np.log(508184 / 100) / np.log(1.01))) < 3


def test_stats_known_answers(known):
    s = known["stats"]
    for c in s["nb_llr"]:
        v = O.nb_llr(*c["args"])
        if c.get("none"):
            assert v is None, c["ref"]
        elif "abs_lt" in c:
            assert abs(v) < c["abs_lt"], c["ref"]
        else:
            assert v > c["gt"], c["ref"]
    for x, want, tol in s["erfc"]["cases"]:
        assert abs(O.erfc(x) - want) < tol
    assert O.erfc(5.0) < s["erfc"]["erfc5_lt"]
    d = s["depleted"]
    q = np.array(d["query"], np.uint32)
    groups = O.query_groups(q[:, 0], q[:, 1])
    mv = np.tile(np.array(d["moments"], np.float32), (2000, 1))  # every slot holds (20, 100)
    p0, _ = O.analytic_stats([(0, groups)], {0: (10**7, mv)}, 0.0)
    assert p0 == d["obs_zero_p"]
    p, llr = O.analytic_stats([(0, groups)], {0: (10**7, mv)}, d["obs_depleted"])
    assert 0.5 < p < 1.0


def test_stats_no_shared_chrom_and_enriched():
    # stats.rs:145-157: query chr21 only, DB chr22 only -> None
    q = O.query_groups(np.array([10_000_000], np.uint32), np.array([10_001_000], np.uint32))
    nb22 = (50_818_468 + 99) // 100
    g = O.depth_signal(np.array([10_000_000], np.uint32), np.array([10_001_000], np.uint32), nb22)
    mv, _, _ = O.moments_from_signal(g)
    assert O.analytic_stats([(21, q)], {22: (nb22, mv)}, 0.0) is None
    # stats.rs:175-193: 500 intervals of 5 kb every 10 kb, self query, observed 25000 bins
    s = (np.arange(500) * 10_000).astype(np.uint32)
    e = s + 5000
    g = O.depth_signal(s, e, nb22)
    mv, _, _ = O.moments_from_signal(g)
    q = O.query_groups(s, e)
    p, llr = O.analytic_stats([(22, q)], {22: (nb22, mv)}, 25_000.0)
    assert llr is None or llr >= 0
    assert p < 0.5
    # stats.rs:159-173: zero observed -> p = 1
    q = O.query_groups(np.array([0], np.uint32), np.array([1_000_000], np.uint32))
    g = O.depth_signal(np.array([49_000_000], np.uint32), np.array([50_000_000], np.uint32), nb22)
    mv, _, _ = O.moments_from_signal(g)
    p, _ = O.analytic_stats([(22, q)], {22: (nb22, mv)}, 0.0)
    assert p == 1.0


def test_query_database_matches_bruteforce():
    import helpers
    import riggle_b200 as rg

    rng = np.random.default_rng(11)
    blocks = []
    for sh in range(3):
        blocks.append((sh, helpers.random_db(rng, 3000, 5_000_000, 7)))
    layers = rg.bucket_layers(blocks)
    qsh = {sh: helpers.queries_touching(rng, b, 400, 5) for sh, b in blocks}
    c1, f32, bp1, st = O.query_database(layers, qsh, 5, 7)
    c2, bp2 = O.bruteforce(layers, qsh, 5, 7)
    assert (c1 == c2).all() and (bp1 == bp2).all()
    np.testing.assert_allclose(f32, bp1 / 100.0, rtol=1e-4)
    c3, _, bp3, _ = O.query_database(layers, qsh, 5, 7, threads=4, mode=1)
    assert (c3 == c1).all() and (bp3 == bp1).all()
    assert st["hits"] == int(c1.sum())


def test_batched_query_matches_unbatched():
    # src/tasks/query/mod.rs:455-499: counts do not depend on how query files are batched
    import helpers
    import riggle_b200 as rg

    rng = np.random.default_rng(3)
    blocks = [(0, helpers.random_db(rng, 2000, 2_000_000, 4))]
    layers = rg.bucket_layers(blocks)
    q = helpers.queries_touching(rng, blocks[0][1], 300, 130)  # 130 rows -> 3 windows of 64
    full, _, bpf, _ = O.query_database(layers, {0: q}, 130, 4, threads=3)
    for r in range(130):
        sub = q[q[:, 2] == r].copy()
        sub[:, 2] = 0
        one, _, bpo, _ = O.query_database(layers, {0: sub}, 1, 4)
        assert (one[0] == full[r]).all() and (bpo[0] == bpf[r]).all()


def test_oracle_workload_generator_equals_the_library_generator():
    """The CPU reference arm builds its inputs with the oracle's restatement of the seeded workload
    generator (so it never loads the GPU library); it must produce the library generator's bits."""
    import riggle_b200 as rg

    assert np.array_equal(O.synth_chrom_lengths(1, 24), rg.synth_chrom_lengths(1, 24))
    assert np.array_equal(O.synth_zipf_sizes(1000, 1.1, 1000, 10_000_000, 2_000_000_000),
                          rg.synth_zipf_sizes(1000, 1.1, 1000, 10_000_000, 2_000_000_000))
    assert np.array_equal(O.synth_loguniform_sizes(4242, 300, 100, 1_000_000),
                          rg.synth_loguniform_sizes(4242, 300, 100, 1_000_000))
    cl = O.synth_chrom_lengths(1, 24)
    sizes = O.synth_zipf_sizes(40, 1.1, 100, 20_000, 200_000)
    o = O.SynthWorkload(2, cl, sizes, broad_fraction=0.05)
    r = rg.SynthSpec(2, cl, sizes, broad_fraction=0.05)
    for c in (0, 7, 23):
        ol, rl = o.chrom_layers(c), r.chrom_layers(c)
        assert ol.keys() == rl.keys()
        for k in ol:
            assert np.array_equal(ol[k][0], rl[k][0]) and np.array_equal(ol[k][1], rl[k][1])
    oq = O.SynthWorkload(5000, cl, [3000, 800], hotspot_fraction=0.1, num_hotspots=8)
    rq = rg.SynthSpec(5000, cl, [3000, 800], hotspot_fraction=0.1, num_hotspots=8)
    for f in range(2):
        for c in (0, 3, 23):
            assert np.array_equal(oq.block(f, c), rq.block(f, c))
