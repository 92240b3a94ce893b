"""Multi-GPU partition of the database by file (column sharding).

Rank r holds the layers of a contiguous range of database files (sources) [b[r], b[r+1]) — built
directly with `Index.synth_columns` or cut from a full index with `Index.select_columns` — and
answers the same query batch for its columns.  Counts, overlap base pairs and p-values of a
(query row, source) cell depend only on that source's intervals and moments, so the ranks never
exchange data while sweeping; the only collective is one all-gather of the ranks' column slices
(NCCL over NVLink on GPUs, gloo on CPUs).  The reference runs on one host and has no counterpart.
"""
import numpy as np


def column_bounds(sizes, parts):
    """Contiguous source ranges with near-equal interval counts: bounds b (parts + 1 entries), rank r
    owns sources [b[r], b[r + 1]).  Each cut is the prefix-sum point nearest to an equal share,
    kept strictly increasing while sources remain so that no rank is left without columns."""
    sizes = np.asarray(sizes, dtype=np.float64)
    n = len(sizes)
    if parts < 1:
        raise ValueError("parts must be >= 1")
    cum = np.concatenate([[0.0], np.cumsum(sizes)])
    b = [0]
    for r in range(1, parts):
        target = cum[-1] * r / parts
        k = int(np.argmin(np.abs(cum - target)))  # nearest prefix-sum point
        lo = min(b[-1] + 1, n)                      # strictly increasing while sources remain
        hi = n - (parts - r)                        # one source left for every later rank
        k = lo if hi < lo else min(max(k, lo), hi)
        b.append(k)
    b.append(n)
    return np.array(b, dtype=np.int64)


def gather_columns(local, bounds, group=None):
    """All-gather of column slices: `local` is this rank's [rows, b[r+1] - b[r]] torch tensor; returns
    the full [rows, b[-1]] matrix on every rank (ranks ordered as the bounds)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    widths = [int(bounds[r + 1] - bounds[r]) for r in range(world)]
    w = max(widths) if widths else 0
    rows = local.shape[0]
    pad = torch.zeros((rows, w), dtype=local.dtype, device=local.device)
    pad[:, :local.shape[1]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:, :widths[r]] for r, p in enumerate(parts)], dim=1)


def host_layers_columns(layers, sid_lo, sid_hi):
    """Host-side column filter of {(shard, layer): (pos, sid)} layers (the CPU mirror of
    Index.select_columns): keeps sids in [sid_lo, sid_hi), rebased to 0, order preserved."""
    out = {}
    for key, (pos, sid) in layers.items():
        keep = (sid >= sid_lo) & (sid < sid_hi)
        if keep.any():
            out[key] = (np.ascontiguousarray(pos[keep]), np.ascontiguousarray(sid[keep] - sid_lo))
    return out
