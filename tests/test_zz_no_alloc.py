"""The allocation-free depth signal (rgl_depth_signal_noalloc) against the allocating entry point.

Callers that cannot allocate device memory during a call (graph capture, their own device-memory
arena, latency-critical loops) use rgl_depth_signal_noalloc: its scratch lives in a fixed static
device array.  Two calls in a row, with different inputs, must each reproduce rgl_depth_signal bit
for bit; the second call must not see the first call's leftovers.  This file is collected last so a
failure here leaves the rest of the suite already run."""
import ctypes as C

import numpy as np
import pytest

import riggle_b200 as rg
from riggle_b200 import _lib, api

pytestmark = pytest.mark.gpu


def _noalloc(iv, n_bins, bin_size=100):
    import torch

    lib = rg.load()
    d_iv = torch.from_numpy(np.ascontiguousarray(iv, np.uint32).view(np.int32)).cuda()
    d_g = torch.full((n_bins,), 7.0, dtype=torch.float32, device="cuda")  # garbage to be overwritten
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.rgl_depth_signal_noalloc(0, C.c_void_p(d_iv.data_ptr()) if len(iv) else None, len(iv), n_bins,
                                            bin_size, C.c_void_p(d_g.data_ptr()), C.c_void_p(stream)))
    torch.cuda.synchronize()
    return d_g.cpu().numpy()


def _intervals(rng, n, span):
    s = rng.integers(0, span, n).astype(np.int64)
    e = s + rng.integers(1, 20_000, n)
    return np.stack([s, e, np.zeros(n)], 1).astype(np.uint32)


def test_noalloc_matches_allocating_entry_point_twice():
    rng = np.random.default_rng(2024)
    first = (_intervals(rng, 50_000, 300_000 * 100), 300_000)  # large call
    second = (_intervals(rng, 700, 40_003 * 100), 40_003)        # smaller call on a dirty array
    for iv, n_bins in (first, second):
        want = api.depth_signal(iv, n_bins)
        got = _noalloc(iv, n_bins)
        assert np.array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    iv = np.zeros((65_537, 3), np.uint32)  # one more than RGL_NOALLOC_MAX_INTERVALS
    iv[:, 1] = 1
    with pytest.raises(rg.RiggleError) as e:
        _noalloc(iv, 1000)
    assert e.value.status == _lib.RGL_ERR_INVALID_ARGUMENT
    with pytest.raises(rg.RiggleError) as e:
        _noalloc(iv[:10], 4_194_305)
    assert e.value.status == _lib.RGL_ERR_INVALID_ARGUMENT


def test_noalloc_refuses_an_output_off_a_16_byte_boundary():
    import torch

    lib = rg.load()
    iv = np.array([[100, 900, 0]], np.uint32)
    d_iv = torch.from_numpy(iv.view(np.int32)).cuda()
    d_g = torch.zeros(1001, dtype=torch.float32, device="cuda")
    st = lib.rgl_depth_signal_noalloc(0, C.c_void_p(d_iv.data_ptr()), 1, 1000, 100, C.c_void_p(d_g.data_ptr() + 4),
                                      None)
    assert st == _lib.RGL_ERR_INVALID_ARGUMENT
    # the aligned buffer still works after the refusal
    got = _noalloc(iv, 1000)
    assert np.array_equal(got, api.depth_signal(iv, 1000))
