"""C-ABI checks that need no GPU: the library loads, exports every entry point include/riggle.h
declares, and its host-side arithmetic matches the oracle."""
import ctypes as C
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


def compiled_layout(name):
    lib = rg.load()
    size, align, nf = C.c_uint64(), C.c_uint64(), C.c_uint32()
    cap = 64
    names = (C.c_char_p * cap)()
    offs = (C.c_uint64 * cap)()
    sizes = (C.c_uint64 * cap)()
    _lib.check(lib.rgl_abi_layout(name.encode(), C.byref(size), C.byref(align), C.byref(nf), names, offs, sizes,
                                  cap))
    fields = [(names[k].decode(), offs[k], sizes[k]) for k in range(nf.value)]
    return size.value, align.value, fields


def public_structs():
    lib = rg.load()
    out, i = [], 0
    while True:
        n = lib.rgl_abi_struct_name(i)
        if n is None:
            return out
        out.append(n.decode())
        i += 1


def header_structs():
    src = open(os.path.join(ROOT, "include", "riggle.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(re.findall(r"typedef struct (\w+) \{", src))


def test_every_header_struct_has_a_compiled_layout():
    assert sorted(public_structs()) == header_structs()


def test_ctypes_mirrors_match_the_compiled_layout():
    """Every ctypes mirror in riggle_b200/_lib.py has the compiled struct's size, field names and
    offsets (a field added to riggle.h and not to the mirror fails here)."""
    for name in public_structs():
        mirror = _lib.MIRRORS[name]
        size, _, fields = compiled_layout(name)
        assert C.sizeof(mirror) == size, name
        got = [(f, getattr(mirror, f).offset, getattr(mirror, f).size) for f, _ in mirror._fields_]
        assert got == fields, name


_RUST_SCALARS = {"u8": 1, "u16": 2, "u32": 4, "u64": 8, "i32": 4, "i64": 8, "f32": 4, "f64": 8, "c_int": 4,
                 "usize": 8}


def _rust_block():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```rust\n(.*?)```", text, flags=re.S)
    assert m, "INTEGRATION.md has no rust block"
    return re.sub(r"//[^\n]*", "", m.group(1))


def _rust_structs(block):
    out = {}
    for m in re.finditer(r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}", block,
                         flags=re.S):
        fields = []
        for decl in m.group(2).split(","):
            decl = decl.strip()
            if not decl:
                continue
            fm = re.match(r"pub (\w+):\s*(.+)$", decl, flags=re.S)
            assert fm, decl
            fields.append((fm.group(1), " ".join(fm.group(2).split())))
        out[m.group(1)] = fields
    return out


def _c_name(rust_name):
    return "rgl_" + re.sub(r"(?<!^)([A-Z])", r"_\1", rust_name[3:]).lower()


def _rust_layout(structs, name, memo):
    """sizeof / alignof / field offsets of a #[repr(C)] Rust struct, by the C layout rules."""
    if name in memo:
        return memo[name]
    off, align, fields = 0, 1, []
    for f, t in structs[name]:
        if t.startswith("*") or t.startswith("Option<unsafe extern") or t.startswith("Option<extern"):
            fs = fa = 8  # raw pointers and nullable function pointers
        elif t in _RUST_SCALARS:
            fs = fa = _RUST_SCALARS[t]
        else:
            fs, fa, _ = _rust_layout(structs, t, memo)
        off = (off + fa - 1) // fa * fa
        fields.append((f, off, fs))
        off += fs
        align = max(align, fa)
    size = (off + align - 1) // align * align
    memo[name] = (size, align, fields)
    return memo[name]


def test_integration_rust_binding_matches_the_compiled_layout():
    """The #[repr(C)] structs of INTEGRATION.md's Rust binding lay out like the compiled structs, and
    its extern block declares only exported functions, with the header's parameter counts."""
    block = _rust_block()
    structs = _rust_structs(block)
    assert {"RglQueryOpts", "RglBatchOpts", "RglServerOpts", "RglRequest", "RglPvalueBatch"} <= set(structs)
    memo = {}
    for rname in structs:
        cname = _c_name(rname)
        size, align, fields = compiled_layout(cname)
        rsize, ralign, rfields = _rust_layout(structs, rname, memo)
        assert (rsize, ralign) == (size, align), rname
        assert rfields == fields, rname
    # every struct named in a function signature is declared in the block (or opaque)
    opaque = set(re.findall(r"pub enum (\w+) \{\}", block))
    for t in set(re.findall(r"\b(Rgl\w+)\b", block)):
        assert t in structs or t in opaque, f"{t} is used but not declared"
    src = open(os.path.join(ROOT, "include", "riggle.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    for m in re.finditer(r"pub fn (rgl_\w+)\((.*?)\)\s*->", block, flags=re.S):
        fn, args = m.group(1), m.group(2).strip()
        hm = re.search(r"\b" + fn + r"\s*\((.*?)\);", src, flags=re.S)
        assert hm, f"{fn} is not declared in riggle.h"
        nc = 0 if hm.group(1).strip() in ("", "void") else hm.group(1).count(",") + 1
        nr = 0 if not args else args.rstrip(",").count(",") + 1
        assert nr == nc, f"{fn}: {nr} parameters in the binding, {nc} in riggle.h"


def test_noalloc_depth_signal_refuses_misaligned_buffers():
    """rgl_depth_signal_noalloc reads and writes d_g as float4 and reads the intervals as u32 words:
    a d_g off a 16-byte boundary or intervals off a 4-byte boundary are refused before anything is
    enqueued (so this runs without a GPU; the pointers are never dereferenced)."""
    lib = rg.load()
    for iv, g in ((0x10000, 0x20004), (0x10000, 0x20008), (0x10002, 0x20000)):
        st = lib.rgl_depth_signal_noalloc(0, C.c_void_p(iv), 10, 1000, 100, C.c_void_p(g), None)
        assert st == _lib.RGL_ERR_INVALID_ARGUMENT
        assert b"aligned" in lib.rgl_last_error()
