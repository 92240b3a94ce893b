"""C-ABI checks that need no GPU: the library loads, exports every entry point include/riggle.h
declares, and its host-side arithmetic matches the oracle."""
import os
import re

import numpy as np
import pytest

import oracle as O
import riggle_b200 as rg
from riggle_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "riggle.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(rgl_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_function():
    lib = rg.load()
    names = header_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) <= set(names)


def test_version_and_status_strings():
    lib = rg.load()
    assert lib.rgl_version() >= 100
    for code in _lib.STATUS_NAMES:
        assert lib.rgl_status_str(code)


def test_layer_config_matches_oracle():
    rng = np.random.default_rng(0)
    for mn, gf in [(128, 4), (100, 3), (1, 2), (256, 2), (7, 5)]:
        lc = rg.LayerConfig(mn, gf)
        for size in list(rng.integers(0, 2**32, 200)) + [0, mn - 1, mn, mn * gf, 2**32 - 1]:
            size = int(size) % 2**32
            assert lc.layer_for_size(size) == O.lib().orc_layer_for_size(mn, gf, size)
        for k in range(20):
            assert lc.layer_max_size(k) == O.lib().orc_layer_max_size(mn, gf, k)
            assert lc.tile_size(k) == O.lib().orc_tile_size(mn, gf, k)


def test_synth_blocks_are_deterministic_and_valid():
    cl = rg.synth_chrom_lengths(1, 24)
    assert cl.min() >= 50_000_000 and cl.max() < 250_000_000
    sp = rg.SynthSpec(2, cl, [50_000, 20_000], broad_fraction=0.05)
    assert sp.chrom_counts(0).sum() == 50_000
    a, b = sp.block(0, 3), sp.block(0, 3)
    assert (a == b).all()
    assert (a[:, 0] < a[:, 1]).all() and (a[:, 1] <= cl[3]).all()
    assert (np.diff(a[:, 0].astype(np.int64)) >= 0).all()
    lens = np.concatenate([sp.block(0, c) for c in range(24)])
    lens = (lens[:, 1] - lens[:, 0]).astype(np.float64)
    narrow = lens[lens <= 100_000]
    assert abs(np.median(narrow) - 500) < 40          # log-normal median 500
    assert 0.03 < np.mean(lens >= 10_000 + 0 * lens) < 0.09  # ~5% broad (+ narrow tail)


def test_zipf_sizes():
    z = rg.synth_zipf_sizes(1000)
    assert abs(int(z.sum()) - 2_000_000_000) < 2_000_000
    assert z.max() == 10_000_000 and z.min() >= 1000
    assert (np.diff(z.astype(np.int64)) <= 0).all()


def test_open_missing_database_is_database_not_found(tmp_path):
    with pytest.raises(rg.RiggleError) as e:
        rg.Index.open(tmp_path / "nope")
    assert e.value.status == _lib.RGL_ERR_DATABASE_NOT_FOUND


def test_bad_meta_json_is_meta_error(tmp_path):
    (tmp_path / "meta.json").write_text("{not json")
    with pytest.raises(rg.RiggleError) as e:
        rg.Index.open(tmp_path)
    assert e.value.status == _lib.RGL_ERR_META_JSON
