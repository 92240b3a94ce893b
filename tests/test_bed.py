"""BED ingest (rgl_bed_*): the reference's parser unit tests (src/io/parse.rs:180-300) and the
file-batch rules of parse_file_batch (src/tasks/query/files.rs:25-111).  Host only, except the last
test, which runs the counting path on a parsed batch."""
import gzip

import numpy as np
import pytest

import riggle_b200 as rg


def parse(text, sid=1):
    b = rg.BedBatch.parse_string(text, sid)
    return b.shards(0)


def test_parse_basic_bed():
    s = parse("chr1\t100\t200\nchr1\t300\t400\n")
    assert list(s) == ["chr1"]
    assert s["chr1"].tolist() == [[100, 200, 1], [300, 400, 1]]


def test_parse_multi_shard():
    s = parse("chr1\t100\t200\nchr2\t300\t400\nchr1\t500\t600\n")
    assert len(s) == 2 and len(s["chr1"]) == 2 and len(s["chr2"]) == 1


def test_parse_extended_bed():
    s = parse("chr1\t100\t200\tpeak1\t500\t+\n", 2)
    assert s["chr1"].tolist() == [[100, 200, 2]]


def test_parse_no_shard_column():
    s = parse("100\t200\n300\t400\n")
    assert list(s) == ["default"] and len(s["default"]) == 2


def test_parse_comments_empty_lines_spaces():
    assert len(parse("# c\nchr1\t100\t200\n# c2\nchr1\t300\t400\n")["chr1"]) == 2
    assert len(parse("chr1\t100\t200\n\n\nchr1\t300\t400\n   \nchr1\t500\t600\n")["chr1"]) == 3
    s = parse("chr1 100 200\nchr1   300   400\n")
    assert s["chr1"][:, 0].tolist() == [100, 300]
    assert parse("chr1\t100\t200\r\n\r\nchr1\t5\t9")["chr1"].tolist() == [[100, 200, 1], [5, 9, 1]]


def test_parse_errors_with_line_numbers():
    with pytest.raises(rg.RiggleError, match=r"BED_INVALID_FORMAT: Line 1:"):
        parse("100\n")
    with pytest.raises(rg.RiggleError, match=r"BED_INVALID_RANGE: Line 1: start \(200\)"):
        parse("chr1\t200\t100\n")
    with pytest.raises(rg.RiggleError, match="BED_INVALID_RANGE"):
        parse("chr1\t100\t100\n")
    with pytest.raises(rg.RiggleError, match=r"BED_INVALID_FORMAT: Line 3:"):
        parse("chr1\t1\t2\n# x\nchr1\tfoo\t7\n")


def test_parse_u32_rules():
    # '+' is accepted; a number past u32 is not an integer and becomes the shard
    assert parse("chr1\t+10\t+20\n")["chr1"].tolist() == [[10, 20, 1]]
    assert parse("4294967296\t5\t9\n")["4294967296"].tolist() == [[5, 9, 1]]
    assert parse("chrX\t4294967294\t4294967295\n")["chrX"].tolist() == [[4294967294, 4294967295, 1]]
    # the first non-integer token names the shard, wherever it is
    assert parse("10\t20\tchr7\n")["chr7"].tolist() == [[10, 20, 1]]


def test_batch_load_sorts_skips_empty_and_compacts(tmp_path):
    (tmp_path / "b.bed").write_text("chr1\t10\t20\nchr2\t5\t6\n")
    (tmp_path / "a.bed").write_text("chr2\t1\t2\n")
    (tmp_path / "c.bed").write_text("# only a comment\n")
    with gzip.open(tmp_path / "d.bed.gz", "wt") as f:
        f.write("chr1\t7\t8\n")
    with open(tmp_path / "d.bed.gz", "ab") as f:  # a second gzip member
        f.write(gzip.compress(b"chr3\t70\t80\n"))
    (tmp_path / "x.txt").write_text("chr1\t1\t2\n")
    b = rg.BedBatch.load(tmp_path, threads=3)
    assert b.rows == 3
    assert [b.name(r) for r in range(3)] == ["a.bed", "b.bed", "d.bed.gz"]
    assert [b.count(r) for r in range(3)] == [1, 2, 2]
    assert b.shards(1)["chr2"].tolist() == [[5, 6, 1]]
    assert list(b.shards(2)) == ["chr1", "chr3"]  # first-appearance order, both gzip members read
    assert b.shards(2)["chr3"].tolist() == [[70, 80, 2]]
    one = rg.BedBatch.load(tmp_path / "b.bed")
    assert one.rows == 1 and one.shards(0)["chr1"].tolist() == [[10, 20, 0]]
    (tmp_path / "e.bed").write_text("chr1\t1\t2\nchr1\t9\t3\n")
    with pytest.raises(rg.RiggleError, match=r"e.bed: Line 2"):
        rg.BedBatch.load(tmp_path)
    with pytest.raises(rg.RiggleError, match="INPUT_NOT_FOUND"):
        rg.BedBatch.load(tmp_path / "missing")


@pytest.mark.gpu
def test_batch_query_equals_query_counts(tmp_path):
    import helpers

    rng = np.random.default_rng(4)
    blocks = [(sh, helpers.random_db(rng, 5000, 1_000_000, 6)) for sh in range(2)]
    layers = rg.bucket_layers(blocks)
    idx = rg.Index.from_layers(layers, 6, ["chr1", "chr2"])
    ctx = rg.Context(idx)
    files = {}
    for i in range(3):
        lines, per = [], {}
        for sh, name in ((0, "chr1"), (1, "chr2"), (None, "chrUn")):
            q = helpers.random_db(rng, 50, 1_000_000, 1)
            lines += [f"{name}\t{s}\t{e}" for s, e, _ in q]
            if sh is not None:
                per[name] = q
        (tmp_path / f"q{i}.bed").write_text("\n".join(lines) + "\n")
        files[i] = per
    b = rg.BedBatch.load(tmp_path)
    c, bp, _ = b.query(ctx)
    qs = {}
    for i, per in files.items():
        for name, q in per.items():
            q = q.copy()
            q[:, 2] = i
            qs.setdefault(name, []).append(q)
    c2, bp2, _ = ctx.query_counts({k: np.concatenate(v) for k, v in qs.items()}, 3)
    assert (c == c2).all() and (bp == bp2).all() and c.sum() > 0
    ctx.close()
    idx.close()
