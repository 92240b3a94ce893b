"""Index build on the device (rgl_index_add_beds) and the writer of the reference's database layout
(rgl_index_write), against the oracle's bucketing, reverse co-merge (extend_layer) and jump table.
Needs a GPU."""
import json

import numpy as np
import pytest

import helpers
import oracle as O
import riggle_b200 as rg

pytestmark = pytest.mark.gpu

CHROMS = ["chr1", "chr2", "chrM"]


def _write_beds(d, rng, nfiles, sid0, with_empty=False):
    """BED files with lengths across the layers and duplicated starts; returns the parsed blocks
    [(shard id, uint32[n,3])] in file (path) order, sid = sid0 + file position."""
    d.mkdir(parents=True, exist_ok=True)
    blocks = []
    names = [f"f{i:02d}.bed" for i in range(nfiles)]
    for i, name in enumerate(names):
        lines = []
        if with_empty and i == 1:
            (d / name).write_text("# nothing here\n")
            continue
        per = {c: [] for c in range(len(CHROMS))}
        n = int(rng.integers(50, 400))
        starts = rng.integers(0, 2_000_000, n)
        starts[: n // 5] = starts[n // 5: 2 * (n // 5)]  # equal starts across and within files
        lens = np.exp(rng.normal(np.log(500), 1.5, n)).astype(np.int64).clip(1, 300_000)
        chrom = rng.integers(0, len(CHROMS), n)
        for s, l, c in zip(starts, lens, chrom):
            lines.append(f"{CHROMS[c]}\t{s}\t{s + l}")
            per[c].append((s, s + l, sid0 + i))
        (d / name).write_text("\n".join(lines) + "\n")
        for c in range(len(CHROMS)):
            if per[c]:
                blocks.append((c, np.array(per[c], np.uint32)))
    return blocks


def _layers_of(idx):
    out = {}
    for sh in range(idx.num_shards):
        for k in range(idx.num_layer_slots):
            if idx.layer_count(sh, k):
                out[(sh, k)] = idx.export_layer(sh, k)
    return out


def test_build_equals_oracle_bucketing_and_query(tmp_path):
    rng = np.random.default_rng(1)
    blocks = _write_beds(tmp_path / "a", rng, 5, 0, with_empty=True)
    idx = rg.Index.from_beds(tmp_path / "a", threads=3)
    assert idx.num_sources == 5  # the empty file keeps its D_SID
    assert idx.source_name(1) == "f01.bed"
    names = [idx.shard_name(s) for s in range(idx.num_shards)]
    assert sorted(names) == sorted(CHROMS)  # ids in first-appearance order over the files
    blocks = [(names.index(CHROMS[c]), b) for c, b in blocks]
    want = rg.bucket_layers(blocks)  # stable by start: file then line order on ties
    got = _layers_of(idx)
    assert set(got) == set(want)
    for k in want:
        assert (got[k][0] == want[k][0]).all() and (got[k][1] == want[k][1]).all(), k
    # queries against it equal an index loaded from the same layers
    ref = rg.Index.from_layers(want, 5, names)
    q = {names[c]: helpers.queries_touching(rng, b, 300, 2) for c, b in blocks[:3]}
    a, abp, _ = rg.Context(idx).query_counts(q, 2)
    b, bbp, _ = rg.Context(ref).query_counts(q, 2)
    assert (a == b).all() and (abp == bbp).all()


def test_add_merges_like_extend_layer(tmp_path):
    rng = np.random.default_rng(2)
    _write_beds(tmp_path / "a", rng, 3, 0)
    base = rg.Index.from_beds(tmp_path / "a")
    new_blocks = _write_beds(tmp_path / "b", rng, 4, 3)
    merged = base.add_beds(tmp_path / "b")
    assert merged.num_sources == 7 and base.num_sources == 3
    names = [merged.shard_name(s) for s in range(merged.num_shards)]
    assert names[:base.num_shards] == [base.shard_name(s) for s in range(base.num_shards)]
    new_layers = rg.bucket_layers([(names.index(CHROMS[c]), b) for c, b in new_blocks])
    old = _layers_of(base)
    got = _layers_of(merged)
    for k in set(old) | set(new_layers):
        if k in old and k in new_layers:
            npos, nsid = new_layers[k]
            ivs = np.concatenate([npos, nsid[:, None]], 1)
            want_pos = np.empty((len(old[k][1]) + len(nsid), 2), np.uint32)
            want_sid = np.empty(len(old[k][1]) + len(nsid), np.uint32)
            O.lib().orc_extend_layer(O._p(old[k][0]), O._p(old[k][1]), len(old[k][1]), O._p(ivs), len(ivs),
                                     O._p(want_pos), O._p(want_sid))
        elif k in old:
            want_pos, want_sid = old[k]
        else:
            want_pos, want_sid = new_layers[k]
        assert (got[k][0] == want_pos).all() and (got[k][1] == want_sid).all(), k


def test_write_round_trip_and_jump_tables(tmp_path):
    rng = np.random.default_rng(3)
    _write_beds(tmp_path / "a", rng, 4, 0)
    idx = rg.Index.from_beds(tmp_path / "a")
    db = tmp_path / "db"
    idx.write(db)
    meta = json.loads((db / "meta.json").read_text())
    assert meta["layer_config"] == {"min_size": 128, "growth_factor": 4}
    assert meta["shards"] == [idx.shard_name(s) for s in range(idx.num_shards)]
    assert meta["sid_map"]["2"] == {"name": "f02.bed"}
    again = rg.Index.open(db)
    a, b = _layers_of(idx), _layers_of(again)
    assert set(a) == set(b)
    for k in a:
        assert (a[k][0] == b[k][0]).all() and (a[k][1] == b[k][1]).all()
        tile = rg.LayerConfig().tile_size(k[1])
        jt = np.fromfile(db / "shards" / idx.shard_name(k[0]) / f"layer_{k[1]}.idx", np.uint64)
        assert (jt == O.build_jump_table(a[k][0][:, 0], tile)).all(), k


def test_add_errors(tmp_path):
    with pytest.raises(rg.RiggleError, match="INPUT_NOT_FOUND"):
        rg.Index.from_beds(tmp_path / "missing")
    (tmp_path / "x.txt").write_text("chr1\t1\t2\n")
    with pytest.raises(rg.RiggleError, match="NO_BED_FILES"):
        rg.Index.from_beds(tmp_path)
    with pytest.raises(rg.RiggleError, match="NO_BED_FILES"):
        rg.Index.from_beds(tmp_path / "x.txt")
    (tmp_path / "bad.bed").write_text("chr1\t5\t5\n")
    with pytest.raises(rg.RiggleError, match="BED_INVALID_RANGE"):
        rg.Index.from_beds(tmp_path)
