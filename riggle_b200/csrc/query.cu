// The sweep: query_database's counting path (src/tasks/query/mod.rs:182-307) and
// query_sweep_windowed (src/sweep/query.rs:127-160) as one device pipeline.
//
// Per batch (all on the context stream, no host synchronisation, graph-capturable once the
// workspace is reserved):
//   1. k_expand_keys: each query interval becomes key (segment << 32 | start), value end, and a
//      second key (segment << 32 | end); segment = shard * rows + Q_SID.  Invalid intervals
//      (start >= end, sid >= rows) raise an error bit.
//   2. radix sort both key sets (the reference sorts by (sid, start), mod.rs:202; ends are sorted
//      too, which the rank formulation below needs).
//   3. exclusive u64 prefix sums of the sorted starts and sorted ends (PS, PE).
//   4. K1 partition: for every (layer slot K, query i) the candidate range of the reference's scan,
//      [pp(start - max_K), pp(end)) with pp = partition point of the layer's starts
//      (src/sweep/query.rs:141-148); a segmented max-scan merges them into disjoint ranges per
//      (K, segment); an exclusive scan of the range lengths lays all ranges end to end.
//   5. K2 sweep (k_sweep): a persistent kernel pulls fixed-size chunks of that concatenated range
//      space from a device counter.  Each thread takes one DB interval d and computes, against the
//      segment's sorted query starts S and ends E,
//          count(d) = #{q : q.start < d.end} - #{q : q.end <= d.start}
//          bp(d)    = Cov(d.end) - Cov(d.start),  Cov(x) = x (S<x - E<=x) - PS(S<x) + PE(E<=x)
//      which equal the number of overlapping query intervals and their summed intersection length
//      whenever every DB interval of layer K is non-empty and shorter than max_K — the size-class
//      invariant the reference's add establishes (src/io/meta.rs:33-58) and index validation checks.
//      Under that invariant the look-back bound q.start - max_K <= d.start of the reference's scan
//      never excludes an overlapping pair, so the counts are the reference's, bit for bit.  All
//      ranks lie inside the window of queries that produced d's range, so the searches are short.
//      Counts and base pairs are tallied per (row, source) in shared memory when a chunk belongs to
//      one row, else with global atomics.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "internal.h"

namespace rgl {

struct RangeDesc {
    uint32_t db_lo, db_hi;      // DB index range within the layer
    uint32_t i_first, i_last;   // queries whose candidate windows formed the range (sorted positions)
    uint32_t layer_idx;         // index into the layer table
    uint32_t qrow;              // query row (Q_SID)
    uint32_t seg;               // query segment (shard, row)
    uint32_t slot;              // layer slot K
};

// One query's candidate run for the pair sweep: DB elements [base, base + plen) of its layer.
struct PairSeg {
    uint64_t base;
    uint32_t qs, qe, qrow, pad;
};

enum : uint8_t { M_RANK = 0, M_PAIR = 1 };

// Rank table of one query segment: bin b (width 2^shift bp) holds, at tab[off + b], the number of
// the segment's sorted starts (tab_s) or ends (tab_e) below b << shift, as absolute positions in
// the sorted arrays.  A rank is then one table read plus a search over at most one bin.
struct SegTab {
    uint32_t beg, end;  // the segment's positions in the sorted arrays
    uint32_t shift, nbins;
    uint32_t off;       // first entry of the segment's tables (nbins + 1 entries each)
    uint32_t pad;
};

struct MaxOp {
    __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

enum : uint32_t { ERR_BAD_INTERVAL = 1u, ERR_BAD_ROW = 2u };

// ---- small device helpers ----------------------------------------------------------------------
__device__ __forceinline__ uint32_t lb_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi, uint32_t x) {
    // first index in [lo, hi) with a[i] >= x
    while (lo < hi) {
        uint32_t m = lo + ((hi - lo) >> 1);
        if (__ldg(a + m) < x) lo = m + 1; else hi = m;
    }
    return lo;
}
__device__ __forceinline__ uint32_t ub_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi, uint32_t x) {
    // first index in [lo, hi) with a[i] > x
    while (lo < hi) {
        uint32_t m = lo + ((hi - lo) >> 1);
        if (__ldg(a + m) <= x) lo = m + 1; else hi = m;
    }
    return lo;
}
__device__ __forceinline__ uint32_t pp_layer(const uint2* __restrict__ pos, uint32_t n, uint32_t x) {
    // partition point of (start < x) over a layer sorted by start
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t m = lo + ((hi - lo) >> 1);
        if (__ldg(&pos[m].x) < x) lo = m + 1; else hi = m;
    }
    return lo;
}

// ---- 1. keys ------------------------------------------------------------------------------------
__global__ void k_expand_keys(uint32_t n, const rgl_interval* __restrict__ iv, const uint64_t* __restrict__ blk_off,
                              const uint32_t* __restrict__ blk_shard, uint32_t nblk, uint32_t rows,
                              uint64_t* __restrict__ key, uint32_t* __restrict__ val, uint64_t* __restrict__ ekey,
                              uint32_t* __restrict__ err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t lo = 0, hi = nblk;  // block b with blk_off[b] <= i < blk_off[b+1]
    while (hi - lo > 1) {
        uint32_t m = (lo + hi) >> 1;
        if (blk_off[m] <= i) lo = m; else hi = m;
    }
    const uint32_t* w = reinterpret_cast<const uint32_t*>(iv) + 3ull * i;
    uint32_t s = w[0], e = w[1], q = w[2];
    uint32_t bad = 0;
    if (s >= e) bad |= ERR_BAD_INTERVAL;
    if (q >= rows) { bad |= ERR_BAD_ROW; q = 0; }
    if (bad) atomicOr(err, bad);
    uint64_t seg = (uint64_t)blk_shard[lo] * rows + q;
    key[i] = (seg << 32) | s;
    val[i] = e;
    ekey[i] = (seg << 32) | e;
}

// ---- 2/3. unpack sorted keys ---------------------------------------------------------------------
__global__ void k_unpack(uint32_t n, const uint64_t* __restrict__ key, const uint64_t* __restrict__ ekey,
                         uint32_t* __restrict__ starts, uint32_t* __restrict__ ends_s, uint32_t* __restrict__ seg,
                         uint32_t* __restrict__ segflag, uint64_t* __restrict__ ps_in, uint64_t* __restrict__ pe_in) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        ps_in[n] = 0;
        pe_in[n] = 0;
        return;
    }
    uint64_t k = key[i], ek = ekey[i];
    uint32_t s = (uint32_t)k, e = (uint32_t)ek;
    uint32_t sg = (uint32_t)(k >> 32);
    starts[i] = s;
    ends_s[i] = e;
    seg[i] = sg;
    segflag[i] = (i == 0 || (uint32_t)(key[i - 1] >> 32) != sg) ? 1u : 0u;
    ps_in[i] = s;
    pe_in[i] = e;
}

__global__ void k_seg_begin(uint32_t n, const uint32_t* __restrict__ segflag, const uint32_t* __restrict__ segnum,
                            uint32_t* __restrict__ seg_begin) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (segflag[i]) seg_begin[segnum[i] - 1] = i;
    if (i == n - 1) seg_begin[segnum[i]] = n;
}

// Bin width per segment: about four bins per query, at least 64 bp; tab_len = nbins + 1.
__global__ void k_seg_tabsize(uint32_t n, const uint32_t* __restrict__ segnum, const uint32_t* __restrict__ seg_begin,
                              const uint32_t* __restrict__ ends_s, SegTab* __restrict__ tabs,
                              uint32_t* __restrict__ tab_len) {
    uint32_t sgi = blockIdx.x * blockDim.x + threadIdx.x;
    if (sgi > n) return;
    const uint32_t nseg = segnum[n - 1];
    if (sgi >= nseg) {
        tab_len[sgi] = 0;
        return;
    }
    const uint32_t beg = seg_begin[sgi], end = seg_begin[sgi + 1];
    const uint64_t extent = (uint64_t)ends_s[end - 1] + 1;  // covers every start and end of the segment
    const uint64_t want = extent / (4ull * (end - beg));
    uint32_t shift = want > 1 ? 63u - __clzll(want) : 0u;
    if (shift < 6) shift = 6;
    if (shift > 31) shift = 31;
    const uint32_t nbins = (uint32_t)(extent >> shift) + 1;
    tabs[sgi] = SegTab{beg, end, shift, nbins, 0, 0};
    tab_len[sgi] = nbins + 1;
}

// One thread per table entry (grid-stride over all segments' entries): the entry's segment is found
// by binary search over the table offsets, then tab_s[b] = #starts < b << shift and
// tab_e[b] = #ends < b << shift within the segment.
__global__ void k_seg_tabfill(uint32_t n, const uint32_t* __restrict__ segnum, SegTab* __restrict__ tabs,
                              const uint32_t* __restrict__ tab_off, const uint32_t* __restrict__ starts,
                              const uint32_t* __restrict__ ends_s, uint32_t* __restrict__ tab_s,
                              uint32_t* __restrict__ tab_e) {
    const uint32_t nseg = segnum[n - 1];
    const uint32_t total = tab_off[nseg];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nseg - 1;  // last segment with tab_off <= e
        while (lo < hi) {
            uint32_t m = (lo + hi + 1) >> 1;
            if (__ldg(tab_off + m) <= e) lo = m; else hi = m - 1;
        }
        const SegTab t = tabs[lo];
        const uint32_t b = e - __ldg(tab_off + lo);
        if (b == 0) tabs[lo].off = e;
        const uint64_t x = (uint64_t)b << t.shift;
        uint32_t rs, re;
        if (x > 0xFFFFFFFFull) {
            rs = re = t.end;
        } else {
            rs = lb_u32(starts, t.beg, t.end, (uint32_t)x);
            re = lb_u32(ends_s, t.beg, t.end, (uint32_t)x);
        }
        tab_s[e] = rs;
        tab_e[e] = re;
    }
}

// ---- 4. K1 partition -----------------------------------------------------------------------------
// lo/hi of the reference's candidate scan for (slot K, query i), layer-major arrays [K][n].
__global__ void k_lohi(uint32_t n, uint32_t nslots, uint32_t rows, const uint32_t* __restrict__ starts,
                       const uint32_t* __restrict__ qend, const uint32_t* __restrict__ seg,
                       const int32_t* __restrict__ slot, const LayerDev* __restrict__ layers,
                       const uint2* __restrict__ pos, uint32_t* __restrict__ lo_out, uint32_t* __restrict__ hi_out) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= (uint64_t)n * nslots) return;
    uint32_t K = (uint32_t)(t / n), i = (uint32_t)(t % n);
    uint32_t shard = seg[i] / rows;
    int32_t li = slot[(uint64_t)shard * nslots + K];
    uint32_t lo = 0, hi = 0;
    if (li >= 0) {
        LayerDev L = layers[li];
        const uint2* p = pos + L.off;
        uint32_t s = starts[i];
        uint32_t back = s >= L.max_size ? s - L.max_size : 0u;  // saturating_sub, query.rs:141
        lo = pp_layer(p, (uint32_t)L.n, back);
        hi = pp_layer(p, (uint32_t)L.n, qend[i]);
        if (hi < lo) hi = lo;
    }
    lo_out[t] = lo;
    hi_out[t] = hi;
}

// Range starts: first query of a segment, or a query whose lo is past every earlier hi.
__global__ void k_range_flags(uint32_t n, uint32_t nslots, uint32_t rows, const uint32_t* __restrict__ seg,
                              const uint32_t* __restrict__ segflag, const int32_t* __restrict__ slot,
                              const uint32_t* __restrict__ lo, const uint32_t* __restrict__ maxhi,
                              uint32_t* __restrict__ rflag) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t total = (uint64_t)n * nslots;
    if (t > total) return;
    if (t == total) {
        rflag[t] = 0;
        return;
    }
    uint32_t K = (uint32_t)(t / n), i = (uint32_t)(t % n);
    uint32_t shard = seg[i] / rows;
    int32_t li = slot[(uint64_t)shard * nslots + K];
    uint32_t f = 0;
    if (li >= 0) f = (segflag[i] || lo[t] >= maxhi[t - 1]) ? 1u : 0u;
    rflag[t] = f;
}

__global__ void k_range_emit(uint32_t n, uint32_t nslots, uint32_t rows, const uint32_t* __restrict__ seg,
                             const uint32_t* __restrict__ segflag, const uint32_t* __restrict__ segnum,
                             const int32_t* __restrict__ slot,
                             const uint32_t* __restrict__ lo, const uint32_t* __restrict__ maxhi,
                             const uint32_t* __restrict__ rflag, const uint32_t* __restrict__ ridx,
                             RangeDesc* __restrict__ ranges) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t total = (uint64_t)n * nslots;
    if (t >= total) return;
    uint32_t K = (uint32_t)(t / n), i = (uint32_t)(t % n);
    uint32_t sg = seg[i];
    int32_t li = slot[(uint64_t)(sg / rows) * nslots + K];
    if (li < 0) return;
    uint32_t f = rflag[t];
    if (!f && ridx[t] == 0) return;  // unreachable: every valid (K, segment) row starts with a flag
    uint32_t r = ridx[t] + f - 1;  // inclusive range index of this element
    if (f) {
        ranges[r].db_lo = lo[t];
        ranges[r].i_first = i;
        ranges[r].layer_idx = (uint32_t)li;
        ranges[r].qrow = sg % rows;
        ranges[r].seg = segnum[i] - 1;
        ranges[r].slot = K;
    }
    bool last = (i + 1 == n) || segflag[i + 1] || rflag[t + 1];
    if (last) {
        ranges[r].i_last = i;
        ranges[r].db_hi = maxhi[t];
    }
}

// Per range: the reference's candidate count (sum over its queries of hi - lo) against the size of
// the union.  Where the two are close (narrow layers) the pair sweep reads each candidate once with
// trivial per-pair work; where candidate windows overlap heavily (broad layers) the rank sweep reads
// each union element once.  rlen = union length of rank ranges (the rank work space), ulen = union
// length of every range (the swept count of the metric).
__global__ void k_range_method(uint64_t cap, uint32_t n, const uint32_t* __restrict__ ridx_total_ptr,
                               const RangeDesc* __restrict__ ranges, const uint64_t* __restrict__ pc,
                               uint32_t pair_ratio, uint8_t* __restrict__ method, uint64_t* __restrict__ rlen,
                               uint64_t* __restrict__ ulen) {
    const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r > cap) return;
    const uint32_t R = *ridx_total_ptr;
    if (r >= R) {
        rlen[r] = 0;
        ulen[r] = 0;
        return;
    }
    const RangeDesc rd = ranges[r];
    const uint64_t len = rd.db_hi - rd.db_lo;
    const uint64_t t0 = (uint64_t)rd.slot * n + rd.i_first, t1 = (uint64_t)rd.slot * n + rd.i_last + 1;
    const uint64_t cand = pc[t1] - pc[t0];
    const uint8_t m = (cand <= (uint64_t)pair_ratio * len) ? M_PAIR : M_RANK;
    method[r] = m;
    rlen[r] = m == M_RANK ? len : 0;
    ulen[r] = len;
}

__global__ void k_cand_len(uint64_t tot, const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi,
                           uint64_t* __restrict__ cl) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t > tot) return;
    cl[t] = t < tot ? (uint64_t)(hi[t] - lo[t]) : 0;
}

// Pair work space: each query of a pair range contributes its candidate run.
__global__ void k_pair_len(uint32_t n, uint32_t nslots, uint32_t rows, const uint32_t* __restrict__ seg,
                           const int32_t* __restrict__ slot, const LayerDev* __restrict__ layers,
                           const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi,
                           const uint32_t* __restrict__ rflag, const uint32_t* __restrict__ ridx,
                           const uint8_t* __restrict__ method, const uint32_t* __restrict__ starts,
                           const uint32_t* __restrict__ qend, uint64_t* __restrict__ plen, PairSeg* __restrict__ psegs) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t tot = (uint64_t)n * nslots;
    if (t > tot) return;
    if (t == tot) {
        plen[t] = 0;
        return;
    }
    const uint32_t K = (uint32_t)(t / n), i = (uint32_t)(t % n);
    const uint32_t sg = seg[i];
    const int32_t li = slot[(uint64_t)(sg / rows) * nslots + K];
    uint64_t len = 0;
    if (li >= 0) {
        const uint32_t r = ridx[t] + rflag[t] - 1;
        if (method[r] == M_PAIR) {
            len = hi[t] - lo[t];
            psegs[t] = PairSeg{layers[li].off + lo[t], starts[i], qend[i], sg % rows, 0};
        }
    }
    plen[t] = len;
}

struct SweepParams {
    const uint64_t* rpos;   // exclusive scan of range lengths, cap+1 entries; rpos[cap] = total
    uint64_t rcap;          // range capacity (entries of rpos minus one)
    const RangeDesc* ranges;
    const LayerDev* layers;
    const uint2* pos;
    const uint32_t* sid;
    const uint32_t* starts;  // sorted (segment, start)
    const uint32_t* ends;    // sorted (segment, end)
    const uint64_t* ps;      // exclusive prefix sums of starts
    const uint64_t* pe;      // exclusive prefix sums of ends
    uint32_t* counts;        // rows x D
    unsigned long long* bp;  // rows x D (may be null)
    uint32_t* queue;         // work counter
    const uint32_t* item_r0; // first range of each work item (items < item_cap)
    const uint64_t* ppos;    // pair work space: exclusive scan of candidate runs, rcap + 1 entries
    const PairSeg* psegs;
    const uint32_t* item_t0; // first run of each pair work item
    const SegTab* segtabs;   // per query segment
    const uint32_t* tab_s;   // rank tables of sorted starts / ends
    const uint32_t* tab_e;
    uint64_t item_cap;
    uint32_t rows, D, chunk;
    int smem_tally;          // 1: one row, shared-memory histograms
};

// Galloping (exponential) search from a lower bound: first index in [lo, hi) with a[i] >= x
// (UPPER = false) or a[i] > x (UPPER = true).  Cost ~2 log2(answer - lo), so a rank found from
// the previous, nearby rank takes one or two probes.
template <bool UPPER>
__device__ __forceinline__ uint32_t gallop(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi, uint32_t x) {
    if (lo >= hi) return lo;
    uint32_t v = __ldg(a + lo);
    if (UPPER ? (v > x) : (v >= x)) return lo;
    uint32_t prev = lo, step = 1, nxt;
    for (;;) {  // invariant: a[prev] is below the bound
        if (step >= hi - prev) {
            nxt = hi;
            break;
        }
        nxt = prev + step;
        v = __ldg(a + nxt);
        if (UPPER ? (v > x) : (v >= x)) break;
        prev = nxt;
        step <<= 1;
    }
    return UPPER ? ub_u32(a, prev + 1, nxt, x) : lb_u32(a, prev + 1, nxt, x);
}

// Last range r in [r, rmax] with rpos[r] <= p (ranges are visited in increasing p).
__device__ __forceinline__ uint32_t range_advance(const uint64_t* __restrict__ rpos, uint32_t r, uint32_t rmax,
                                                  uint64_t p) {
    if (r >= rmax || __ldg(rpos + r + 1) > p) return r;
    uint32_t lo = r + 1, step = 1, hi;
    for (;;) {  // invariant: rpos[lo] <= p
        if (step > rmax - lo) {
            hi = rmax;
            break;
        }
        hi = lo + step;
        if (__ldg(rpos + hi) > p) {
            hi--;
            break;
        }
        lo = hi;
        step <<= 1;
    }
    while (lo < hi) {  // last m in [lo, hi] with rpos[m] <= p
        uint32_t m = (lo + hi + 1) >> 1;
        if (__ldg(rpos + m) <= p) lo = m; else hi = m - 1;
    }
    return lo;
}

// Work-item partition: item i covers positions [i * chunk, (i + 1) * chunk) of the concatenated
// ranges; item_r0[i] = the range holding its first position (last r with rpos[r] <= i * chunk),
// found by binary search over the range offsets (grid-stride over items).
__global__ void k_item_ranges(uint64_t rcap, const uint64_t* __restrict__ rpos, uint32_t chunk, uint64_t item_cap,
                              uint32_t* __restrict__ item_r0) {
    const uint64_t total = rpos[rcap];
    const uint64_t items = min((total + chunk - 1) / chunk, item_cap);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < items; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = i * chunk;
        uint64_t lo = 0, hi = rcap;
        while (lo < hi) {
            uint64_t m = (lo + hi + 1) >> 1;
            if (__ldg(rpos + m) <= p) lo = m; else hi = m - 1;
        }
        item_r0[i] = (uint32_t)lo;
    }
}

// A lane's position in the range list, with the range's descriptor cached in registers.
struct Cursor {
    uint32_t r;
    uint64_t rlo, rhi;  // [rpos[r], rpos[r + 1])
    RangeDesc rd;
    uint64_t base;      // element offset of the range's first DB interval in the index arrays
    SegTab tab;         // rank table of the range's query segment
};

__device__ __forceinline__ void cursor_load(const SweepParams& P, Cursor& c, uint32_t r) {
    c.r = r;
    c.rlo = __ldg(P.rpos + r);
    c.rhi = __ldg(P.rpos + r + 1);
    c.rd = P.ranges[r];
    c.base = P.layers[c.rd.layer_idx].off + c.rd.db_lo;
    c.tab = P.segtabs[c.rd.seg];
}

// #starts < x and #ends <= x within the cursor's segment, as absolute sorted positions.
__device__ __forceinline__ uint32_t rank_start(const SweepParams& P, const SegTab& t, uint32_t x) {
    const uint32_t b = x >> t.shift;
    if (b >= t.nbins) return t.end;
    const uint32_t lo = __ldg(P.tab_s + t.off + b), hi = __ldg(P.tab_s + t.off + b + 1);
    return lo == hi ? lo : lb_u32(P.starts, lo, hi, x);
}
__device__ __forceinline__ uint32_t rank_end(const SweepParams& P, const SegTab& t, uint32_t x) {
    const uint32_t b = x >> t.shift;
    if (b >= t.nbins) return t.end;
    const uint32_t lo = __ldg(P.tab_e + t.off + b), hi = __ldg(P.tab_e + t.off + b + 1);
    return lo == hi ? lo : ub_u32(P.ends, lo, hi, x);
}

__device__ __forceinline__ void cursor_seek(const SweepParams& P, Cursor& c, uint64_t p) {
    if (p >= c.rhi) cursor_load(P, c, range_advance(P.rpos, c.r, (uint32_t)P.rcap, p));
}

// Base pairs and tally of one DB interval d with a non-zero count (el_s, sl_e already known).
template <bool WITH_BP>
__device__ __forceinline__ void finish_hit(const SweepParams& P, const SegTab& t, uint32_t qrow, uint2 d,
                                          uint32_t sid, uint32_t cnt, uint32_t el_s, uint32_t sl_e,
                                          uint32_t* s_cnt, unsigned long long* s_bp) {
    unsigned long long bpv = 0;
    if (WITH_BP) {
        const uint32_t sl_s = rank_start(P, t, d.x);
        const uint32_t el_e = rank_end(P, t, d.y);
        if (sl_e == sl_s && el_e == el_s) {
            // no query starts or ends inside d: every overlapping query covers all of d
            bpv = (unsigned long long)(d.y - d.x) * cnt;
        } else {
            const unsigned long long ce = (unsigned long long)d.y * (unsigned long long)(sl_e - el_e) -
                                          __ldg(P.ps + sl_e) + __ldg(P.pe + el_e);
            const unsigned long long cs = (unsigned long long)d.x * (unsigned long long)(sl_s - el_s) -
                                          __ldg(P.ps + sl_s) + __ldg(P.pe + el_s);
            bpv = ce - cs;
        }
    }
    if (P.smem_tally) {
        atomicAdd(&s_cnt[sid], cnt);
        if (WITH_BP) atomicAdd(&s_bp[sid], bpv);
    } else {
        const uint64_t cell = (uint64_t)qrow * P.D + sid;
        atomicAdd(&P.counts[cell], cnt);
        if (WITH_BP) atomicAdd(&P.bp[cell], bpv);
    }
}

// Two table entries tab[b], tab[b + 1] (b < nbins) for the bin of x, or (end, end) past the table.
__device__ __forceinline__ uint2 bin_bounds(const uint32_t* __restrict__ tab, const SegTab& t, uint32_t x) {
    const uint32_t b = x >> t.shift;
    if (b >= t.nbins) return make_uint2(t.end, t.end);
    return make_uint2(__ldg(tab + t.off + b), __ldg(tab + t.off + b + 1));
}

constexpr uint32_t kUnroll = 4;  // DB intervals per lane per step

template <bool WITH_BP>
__global__ void __launch_bounds__(256, 3) k_sweep(SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long* s_bp = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + (WITH_BP ? (size_t)P.D * 8 : 0));
    const uint32_t lane = threadIdx.x & 31u;

    const uint64_t total = P.rpos[P.rcap];
    if (P.smem_tally) {
        for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
            s_cnt[k] = 0;
            if (WITH_BP) s_bp[k] = 0;
        }
    }
    __syncthreads();
    // Warps pull work items independently (no block-wide barrier inside the loop).  A step covers
    // 32 * kUnroll consecutive positions; lane l takes positions pb + l + 32 j, so every load of the
    // DB arrays is coalesced, and the kUnroll DB intervals of a lane and their rank-table entries
    // are all requested before any of them is used.  count(d) = #{q.start < d.end} -
    // #{q.end <= d.start} needs two ranks, each one rank-table read plus, rarely, a search inside
    // one bin.
    for (;;) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(P.queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        const uint64_t p0 = (uint64_t)item * P.chunk;
        if (p0 >= total) break;
        const uint64_t p1 = min(p0 + P.chunk, total);
        uint32_t r0;
        if (item < P.item_cap) {
            r0 = __ldg(P.item_r0 + item);
        } else {
            uint64_t lo = 0, hi = P.rcap;
            while (lo < hi) { uint64_t m = (lo + hi + 1) >> 1; if (__ldg(P.rpos + m) <= p0) lo = m; else hi = m - 1; }
            r0 = (uint32_t)lo;
        }
        Cursor c;
        cursor_load(P, c, r0);
        for (uint64_t pb = p0 + lane; pb < p1; pb += 32 * kUnroll) {
            const uint64_t plast = min(pb + 32 * (kUnroll - 1), p1 - 1 - ((p1 - 1 - pb) & 31));
            cursor_seek(P, c, pb);
            if (plast < c.rhi) {
                // all of this lane's positions of the step lie in one range: batch the loads
                const SegTab t = c.tab;
                const uint64_t off = c.base - c.rlo;
                uint2 d[kUnroll];
                uint32_t sid[kUnroll];
#pragma unroll
                for (uint32_t j = 0; j < kUnroll; j++) {
                    const uint64_t pj = pb + 32 * j;
                    if (pj < p1) {
                        d[j] = __ldg(P.pos + off + pj);
                        sid[j] = __ldg(P.sid + off + pj);
                    } else {
                        d[j] = make_uint2(0, 0);
                        sid[j] = 0;
                    }
                }
                uint2 be[kUnroll], bs[kUnroll];
#pragma unroll
                for (uint32_t j = 0; j < kUnroll; j++) {
                    be[j] = bin_bounds(P.tab_e, t, d[j].x);
                    bs[j] = bin_bounds(P.tab_s, t, d[j].y);
                }
#pragma unroll
                for (uint32_t j = 0; j < kUnroll; j++) {
                    if (pb + 32 * j >= p1) continue;
                    const uint32_t el_s = be[j].x == be[j].y ? be[j].x : ub_u32(P.ends, be[j].x, be[j].y, d[j].x);
                    const uint32_t sl_e = bs[j].x == bs[j].y ? bs[j].x : lb_u32(P.starts, bs[j].x, bs[j].y, d[j].y);
                    const uint32_t cnt = sl_e - el_s;
                    if (cnt) finish_hit<WITH_BP>(P, t, c.rd.qrow, d[j], sid[j], cnt, el_s, sl_e, s_cnt, s_bp);
                }
            } else {
                // the step crosses a range boundary: one position at a time
                for (uint64_t pj = pb; pj < p1 && pj <= pb + 32 * (kUnroll - 1); pj += 32) {
                    cursor_seek(P, c, pj);
                    const uint64_t di = c.base + (pj - c.rlo);
                    const uint2 d = __ldg(P.pos + di);
                    const uint32_t el_s = rank_end(P, c.tab, d.x);
                    const uint32_t sl_e = rank_start(P, c.tab, d.y);
                    const uint32_t cnt = sl_e - el_s;
                    if (cnt) finish_hit<WITH_BP>(P, c.tab, c.rd.qrow, d, __ldg(P.sid + di), cnt, el_s, sl_e, s_cnt, s_bp);
                }
            }
        }
    }
    if (P.smem_tally) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
            if (s_cnt[k]) atomicAdd(&P.counts[k], s_cnt[k]);
            if (WITH_BP && s_bp[k]) atomicAdd(&P.bp[k], s_bp[k]);
        }
    }
}

// The pair sweep: the reference's scan (src/sweep/query.rs:147-158) over the candidate runs of the
// queries of pair ranges, every candidate read once by one lane (lane l of a warp takes positions
// p0 + l, p0 + l + 32, ...; consecutive positions of a run are consecutive DB elements, so the loads
// coalesce).  A candidate d of query q overlaps when d.end > q.start (d.start < q.end and the
// look-back bound hold by construction of the run); it adds 1 and min(ends) - max(starts).
template <bool WITH_BP>
__global__ void __launch_bounds__(256, 4) k_pairs(SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long* s_bp = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + (WITH_BP ? (size_t)P.D * 8 : 0));
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t total = P.ppos[P.rcap];
    if (P.smem_tally)
        for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
            s_cnt[k] = 0;
            if (WITH_BP) s_bp[k] = 0;
        }
    __syncthreads();
    for (;;) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(P.queue, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        const uint64_t p0 = (uint64_t)item * P.chunk;
        if (p0 >= total) break;
        const uint64_t p1 = min(p0 + P.chunk, total);
        uint32_t t;
        if (item < P.item_cap) {
            t = __ldg(P.item_t0 + item);
        } else {
            uint64_t lo = 0, hi = P.rcap;
            while (lo < hi) { uint64_t m = (lo + hi + 1) >> 1; if (__ldg(P.ppos + m) <= p0) lo = m; else hi = m - 1; }
            t = (uint32_t)lo;
        }
        uint64_t rlo = __ldg(P.ppos + t), rhi = __ldg(P.ppos + t + 1);
        PairSeg ps = P.psegs[t];
        for (uint64_t p = p0 + lane; p < p1; p += 32) {
            if (p >= rhi) {
                t = range_advance(P.ppos, t, (uint32_t)P.rcap, p);
                rlo = __ldg(P.ppos + t);
                rhi = __ldg(P.ppos + t + 1);
                ps = P.psegs[t];
            }
            const uint64_t di = ps.base + (p - rlo);
            const uint2 d = __ldg(P.pos + di);
            if (d.y > ps.qs) {
                const uint32_t sid = __ldg(P.sid + di);
                if (P.smem_tally) {
                    atomicAdd(&s_cnt[sid], 1u);
                    if (WITH_BP) atomicAdd(&s_bp[sid], (unsigned long long)(min(ps.qe, d.y) - max(ps.qs, d.x)));
                } else {
                    const uint64_t cell = (uint64_t)ps.qrow * P.D + sid;
                    atomicAdd(&P.counts[cell], 1u);
                    if (WITH_BP) atomicAdd(&P.bp[cell], (unsigned long long)(min(ps.qe, d.y) - max(ps.qs, d.x)));
                }
            }
        }
    }
    if (P.smem_tally) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
            if (s_cnt[k]) atomicAdd(&P.counts[k], s_cnt[k]);
            if (WITH_BP && s_bp[k]) atomicAdd(&P.bp[k], s_bp[k]);
        }
    }
}

}  // namespace rgl

using namespace rgl;

// ================================================================================================
// Context
// ================================================================================================
struct rgl_context {
    rgl_index* idx = nullptr;  // holds one reference of the index
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 148;
    DevBuf iv, blk_off, blk_shard, key_a, key_b, val_a, val_b, ekey_a, ekey_b;
    DevBuf starts, ends, seg, segflag, segnum, seg_begin, ps_in, pe_in, ps, pe;
    DevBuf lo, hi, maxhi, rflag, ridx, ranges, rlen, rpos, cub_tmp, small, out_counts, out_bp, item_r0;
    DevBuf segtab, tab_len, tab_off, tab_s, tab_e;
    DevBuf cl, pc, method, ulen, plen, ppos, psegs, item_t0;
    uint32_t* h_small = nullptr;  // pinned mirror of `small`
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t res_n = 0;
    uint32_t res_rows = 0;
    // sweep-kernel timing on the launch stream (rgl_context_set_timing)
    bool timing = false;
    std::vector<cudaEvent_t> tev;  // pairs (start, end)
    size_t tev_used = 0;
    // state of the last launch, for stats
    uint64_t last_tot = 0;
    uint32_t last_launches = 0;
    uint32_t last_n = 0;
};

namespace {

// Work items whose first range is precomputed; items beyond it search the range list themselves.
constexpr uint64_t kItemCap = 1ull << 22;

int ensure_workspace(rgl_context* c, uint64_t n, uint32_t rows, uint32_t nblk) {
    rgl_index* idx = c->idx;
    const uint64_t ns = std::max<uint32_t>(idx->num_slots, 1);
    const uint64_t tot = n * ns;
    RGL_TRY(c->iv.ensure(n * sizeof(rgl_interval) + 16));
    RGL_TRY(c->blk_off.ensure((nblk + 1) * 8ull));
    RGL_TRY(c->blk_shard.ensure((nblk + 1) * 4ull));
    RGL_TRY(c->key_a.ensure(n * 8 + 8));
    RGL_TRY(c->key_b.ensure(n * 8 + 8));
    RGL_TRY(c->val_a.ensure(n * 4 + 4));
    RGL_TRY(c->val_b.ensure(n * 4 + 4));
    RGL_TRY(c->ekey_a.ensure(n * 8 + 8));
    RGL_TRY(c->ekey_b.ensure(n * 8 + 8));
    RGL_TRY(c->starts.ensure(n * 4 + 4));
    RGL_TRY(c->ends.ensure(n * 4 + 4));
    RGL_TRY(c->seg.ensure(n * 4 + 4));
    RGL_TRY(c->segflag.ensure(n * 4 + 4));
    RGL_TRY(c->segnum.ensure(n * 4 + 4));
    RGL_TRY(c->seg_begin.ensure(n * 4 + 4));
    RGL_TRY(c->ps_in.ensure(n * 8 + 16));
    RGL_TRY(c->pe_in.ensure(n * 8 + 16));
    RGL_TRY(c->ps.ensure(n * 8 + 16));
    RGL_TRY(c->pe.ensure(n * 8 + 16));
    RGL_TRY(c->lo.ensure(tot * 4 + 4));
    RGL_TRY(c->hi.ensure(tot * 4 + 4));
    RGL_TRY(c->maxhi.ensure(tot * 4 + 4));
    RGL_TRY(c->rflag.ensure(tot * 4 + 8));
    RGL_TRY(c->ridx.ensure(tot * 4 + 8));
    RGL_TRY(c->ranges.ensure(tot * sizeof(RangeDesc) + sizeof(RangeDesc)));
    RGL_TRY(c->rlen.ensure(tot * 8 + 16));
    RGL_TRY(c->rpos.ensure(tot * 8 + 16));
    RGL_TRY(c->small.ensure(256));
    RGL_TRY(c->item_r0.ensure(kItemCap * 4));
    RGL_TRY(c->item_t0.ensure(kItemCap * 4));
    RGL_TRY(c->cl.ensure(tot * 8 + 16));
    RGL_TRY(c->pc.ensure(tot * 8 + 16));
    RGL_TRY(c->method.ensure(tot + 16));
    RGL_TRY(c->ulen.ensure(tot * 8 + 16));
    RGL_TRY(c->plen.ensure(tot * 8 + 16));
    RGL_TRY(c->ppos.ensure(tot * 8 + 16));
    RGL_TRY(c->psegs.ensure(tot * sizeof(PairSeg) + sizeof(PairSeg)));
    RGL_TRY(c->segtab.ensure((n + 1) * sizeof(SegTab)));
    RGL_TRY(c->tab_len.ensure((n + 2) * 4));
    RGL_TRY(c->tab_off.ensure((n + 2) * 4));
    RGL_TRY(c->tab_s.ensure((10 * n + 16) * 4));
    RGL_TRY(c->tab_e.ensure((10 * n + 16) * 4));
    // CUB temporary storage: the maximum over every primitive used, at these sizes.
    size_t need = 0, b = 0;
    int nn = (int)std::max<uint64_t>(n, 1);
    int nt = (int)std::max<uint64_t>(tot + 1, 1);
    cub::DeviceRadixSort::SortPairs(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, (uint32_t*)nullptr,
                                    (uint32_t*)nullptr, nn, 0, 64, c->stream);
    need = std::max(need, b);
    cub::DeviceRadixSort::SortKeys(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nn, 0, 64, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::InclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, nn, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nn + 1, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::InclusiveScanByKey(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                        MaxOp(), nn, cub::Equality(), c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, nn + 1, c->stream);
    need = std::max(need, b);
    cub::DeviceReduce::Sum(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    RGL_TRY(c->cub_tmp.ensure(need + 256));
    if (rows) {
        RGL_TRY(c->out_counts.ensure((uint64_t)rows * idx->num_sources * 4 + 16));
        RGL_TRY(c->out_bp.ensure((uint64_t)rows * idx->num_sources * 8 + 16));
    }
    c->res_n = std::max(c->res_n, n);
    c->res_rows = std::max(c->res_rows, rows);
    return RGL_OK;
}

inline unsigned grid_for(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

struct Launch {
    uint32_t chunk, ctas_per_sm, block, pair_ratio;
};

Launch pick_launch(const rgl_query_opts* o) {
    Launch l{2048, 4, 256, 2};
    if (o) {
        if (o->chunk) l.chunk = o->chunk;
        if (o->ctas_per_sm) l.ctas_per_sm = o->ctas_per_sm;
        if (o->block) l.block = 256;  // the kernel is compiled for 256 threads
        if (o->pair_ratio) l.pair_ratio = o->pair_ratio;
    }
    l.chunk = (l.chunk + 31) & ~31u;  // keep warps whole
    if (l.chunk < 32) l.chunk = 32;
    if (l.ctas_per_sm < 1) l.ctas_per_sm = 1;
    if (l.ctas_per_sm > 8) l.ctas_per_sm = 8;
    return l;
}

int timing_record(rgl_context* c, bool start) {
    if (start) {
        while (c->tev.size() < 2 * (c->tev_used + 1)) {
            cudaEvent_t e;
            RGL_CUDA(cudaEventCreate(&e));
            c->tev.push_back(e);
        }
        RGL_CUDA(cudaEventRecord(c->tev[2 * c->tev_used], c->stream));
    } else {
        RGL_CUDA(cudaEventRecord(c->tev[2 * c->tev_used + 1], c->stream));
        c->tev_used++;
    }
    return RGL_OK;
}

// After the stream has been synchronised: error bits and stats of the last launch.
int finish(rgl_context* c, const Launch& L, rgl_query_stats* stats) {
    if (stats) {
        float t_sweep = 0, t_all = 0;
        if (c->last_n) {  // the events are recorded only when the pipeline ran
            RGL_CUDA(cudaEventElapsedTime(&t_sweep, c->ev[1], c->ev[2]));
            RGL_CUDA(cudaEventElapsedTime(&t_all, c->ev[0], c->ev[2]));
        }
        stats->query_intervals = c->last_n;
        stats->ranges = c->last_n ? c->h_small[2] : 0;
        uint64_t T = 0;
        if (c->last_n) std::memcpy(&T, c->h_small + 4, 8);
        stats->db_swept = T;
        uint64_t TR = 0, TP = 0;
        if (c->last_n) {
            std::memcpy(&TR, c->h_small + 6, 8);
            std::memcpy(&TP, c->h_small + 8, 8);
        }
        stats->rank_positions = TR;
        stats->pair_candidates = TP;
        stats->work_items = (TR + L.chunk - 1) / L.chunk + (TP + L.chunk - 1) / L.chunk;
        stats->sweep_ms = c->last_n ? t_sweep : 0.f;
        stats->device_ms = c->last_n ? t_all : 0.f;
        stats->chunk = L.chunk;
        stats->ctas_per_sm = L.ctas_per_sm;
        stats->block = L.block;
        stats->kernel_launches = c->last_launches;
    }
    if (c->h_small[0] & ERR_BAD_INTERVAL) return fail(RGL_ERR_INVALID_ARGUMENT, "a query interval has start >= end");
    if (c->h_small[0] & ERR_BAD_ROW) return fail(RGL_ERR_INVALID_ARGUMENT, "a query interval's sid >= num_rows");
    return RGL_OK;
}

// Runs steps 1-5 for n intervals already in c->iv with block table in c->blk_off/c->blk_shard.
int run_pipeline(rgl_context* c, uint64_t n64, uint32_t rows, uint32_t nblk, const rgl_query_opts* opts,
                 uint32_t* d_counts, unsigned long long* d_bp, rgl_query_stats* stats) {
    rgl_index* idx = c->idx;
    cudaStream_t st = c->stream;
    const uint32_t D = idx->num_sources;
    const uint32_t ns = idx->num_slots;
    const uint32_t n = (uint32_t)n64;
    Launch L = pick_launch(opts);
    const bool with_bp = d_bp != nullptr && !(opts && (opts->flags & RGL_QF_NO_OVERLAP));

    uint32_t* d_small = c->small.as<uint32_t>();  // [0] error bits, [1] queue, [2..] scratch
    RGL_CUDA(cudaMemsetAsync(d_small, 0, 64, st));
    if (d_counts) RGL_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)rows * D * 4, st));
    if (d_bp) RGL_CUDA(cudaMemsetAsync(d_bp, 0, (size_t)rows * D * 8, st));
    if (n == 0 || ns == 0) {
        c->last_n = 0;
        c->last_tot = 0;
        c->last_launches = 0;
        if (stats) std::memset(stats, 0, sizeof(*stats));
        RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
        return RGL_OK;
    }
    // key width: segment = shard * rows + row
    uint64_t nseg = (uint64_t)idx->num_shards * rows;
    int segbits = 1;
    while (segbits < 32 && (1ull << segbits) < nseg) segbits++;
    if (nseg >= (1ull << 32)) return fail(RGL_ERR_INVALID_ARGUMENT, "num_shards * num_rows must be < 2^32");

    if (stats) RGL_CUDA(cudaEventRecord(c->ev[0], st));
    uint32_t launches = 0;
    k_expand_keys<<<grid_for(n, 256), 256, 0, st>>>(n, c->iv.as<rgl_interval>(), c->blk_off.as<uint64_t>(),
                                                    c->blk_shard.as<uint32_t>(), nblk, rows, c->key_a.as<uint64_t>(),
                                                    c->val_a.as<uint32_t>(), c->ekey_a.as<uint64_t>(), d_small);
    launches++;
    size_t tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tb, c->key_a.as<uint64_t>(), c->key_b.as<uint64_t>(),
                                             c->val_a.as<uint32_t>(), c->val_b.as<uint32_t>(), (int)n, 0,
                                             32 + segbits, st));
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceRadixSort::SortKeys(c->cub_tmp.p, tb, c->ekey_a.as<uint64_t>(), c->ekey_b.as<uint64_t>(),
                                            (int)n, 0, 32 + segbits, st));
    k_unpack<<<grid_for(n + 1, 256), 256, 0, st>>>(n, c->key_b.as<uint64_t>(), c->ekey_b.as<uint64_t>(),
                                                   c->starts.as<uint32_t>(), c->ends.as<uint32_t>(),
                                                   c->seg.as<uint32_t>(), c->segflag.as<uint32_t>(),
                                                   c->ps_in.as<uint64_t>(), c->pe_in.as<uint64_t>());
    launches++;
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::InclusiveSum(c->cub_tmp.p, tb, c->segflag.as<uint32_t>(), c->segnum.as<uint32_t>(),
                                           (int)n, st));
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->ps_in.as<uint64_t>(), c->ps.as<uint64_t>(),
                                           (int)n + 1, st));
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->pe_in.as<uint64_t>(), c->pe.as<uint64_t>(),
                                           (int)n + 1, st));
    // rank tables of every query segment
    k_seg_begin<<<grid_for(n, 256), 256, 0, st>>>(n, c->segflag.as<uint32_t>(), c->segnum.as<uint32_t>(),
                                                  c->seg_begin.as<uint32_t>());
    k_seg_tabsize<<<grid_for(n + 1, 256), 256, 0, st>>>(n, c->segnum.as<uint32_t>(), c->seg_begin.as<uint32_t>(),
                                                        c->ends.as<uint32_t>(), c->segtab.as<SegTab>(),
                                                        c->tab_len.as<uint32_t>());
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->tab_len.as<uint32_t>(), c->tab_off.as<uint32_t>(),
                                           (int)n + 1, st));
    k_seg_tabfill<<<(unsigned)std::min<uint64_t>((10 * n + 255) / 256, (uint64_t)c->num_sms * 16), 256, 0, st>>>(
        n, c->segnum.as<uint32_t>(), c->segtab.as<SegTab>(), c->tab_off.as<uint32_t>(), c->starts.as<uint32_t>(),
        c->ends.as<uint32_t>(), c->tab_s.as<uint32_t>(), c->tab_e.as<uint32_t>());
    launches += 3;
    const uint64_t tot = (uint64_t)n * ns;
    k_lohi<<<grid_for(tot, 256), 256, 0, st>>>(n, ns, rows, c->starts.as<uint32_t>(), c->val_b.as<uint32_t>(),
                                                c->seg.as<uint32_t>(), idx->d_slot, idx->d_layers, idx->d_pos,
                                                c->lo.as<uint32_t>(), c->hi.as<uint32_t>());
    launches++;
    for (uint32_t K = 0; K < ns; K++) {
        tb = c->cub_tmp.cap;
        RGL_CUDA(cub::DeviceScan::InclusiveScanByKey(c->cub_tmp.p, tb, c->segnum.as<uint32_t>(),
                                                     c->hi.as<uint32_t>() + (uint64_t)K * n,
                                                     c->maxhi.as<uint32_t>() + (uint64_t)K * n, MaxOp(), (int)n,
                                                     cub::Equality(), st));
    }
    k_range_flags<<<grid_for(tot + 1, 256), 256, 0, st>>>(n, ns, rows, c->seg.as<uint32_t>(),
                                                          c->segflag.as<uint32_t>(), idx->d_slot,
                                                          c->lo.as<uint32_t>(), c->maxhi.as<uint32_t>(),
                                                          c->rflag.as<uint32_t>());
    launches++;
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->rflag.as<uint32_t>(), c->ridx.as<uint32_t>(),
                                           (int)(tot + 1), st));
    k_range_emit<<<grid_for(tot, 256), 256, 0, st>>>(n, ns, rows, c->seg.as<uint32_t>(), c->segflag.as<uint32_t>(),
                                                     c->segnum.as<uint32_t>(), idx->d_slot, c->lo.as<uint32_t>(), c->maxhi.as<uint32_t>(),
                                                     c->rflag.as<uint32_t>(), c->ridx.as<uint32_t>(),
                                                     c->ranges.as<RangeDesc>());
    launches++;
    // candidate counts per (K, query) -> per-range method; rank and pair work spaces
    k_cand_len<<<grid_for(tot + 1, 256), 256, 0, st>>>(tot, c->lo.as<uint32_t>(), c->hi.as<uint32_t>(),
                                                       c->cl.as<uint64_t>());
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->cl.as<uint64_t>(), c->pc.as<uint64_t>(),
                                           (int)(tot + 1), st));
    k_range_method<<<grid_for(tot + 1, 256), 256, 0, st>>>(tot, n, c->ridx.as<uint32_t>() + tot,
                                                           c->ranges.as<RangeDesc>(), c->pc.as<uint64_t>(),
                                                           L.pair_ratio, c->method.as<uint8_t>(),
                                                           c->rlen.as<uint64_t>(), c->ulen.as<uint64_t>());
    k_pair_len<<<grid_for(tot + 1, 256), 256, 0, st>>>(n, ns, rows, c->seg.as<uint32_t>(), idx->d_slot,
                                                       idx->d_layers, c->lo.as<uint32_t>(), c->hi.as<uint32_t>(),
                                                       c->rflag.as<uint32_t>(), c->ridx.as<uint32_t>(),
                                                       c->method.as<uint8_t>(), c->starts.as<uint32_t>(),
                                                       c->val_b.as<uint32_t>(), c->plen.as<uint64_t>(),
                                                       c->psegs.as<PairSeg>());
    launches += 3;
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->rlen.as<uint64_t>(), c->rpos.as<uint64_t>(),
                                           (int)(tot + 1), st));
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->plen.as<uint64_t>(), c->ppos.as<uint64_t>(),
                                           (int)(tot + 1), st));
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceReduce::Sum(c->cub_tmp.p, tb, c->ulen.as<uint64_t>(),
                                    reinterpret_cast<uint64_t*>(d_small + 4), (int)tot, st));
    k_item_ranges<<<(unsigned)(c->num_sms * 8), 256, 0, st>>>(tot, c->rpos.as<uint64_t>(), L.chunk, kItemCap,
                                                               c->item_r0.as<uint32_t>());
    k_item_ranges<<<(unsigned)(c->num_sms * 8), 256, 0, st>>>(tot, c->ppos.as<uint64_t>(), L.chunk, kItemCap,
                                                               c->item_t0.as<uint32_t>());
    launches += 2;
    SweepParams P;
    P.item_r0 = c->item_r0.as<uint32_t>();
    P.item_t0 = c->item_t0.as<uint32_t>();
    P.ppos = c->ppos.as<uint64_t>();
    P.psegs = c->psegs.as<PairSeg>();
    P.segtabs = c->segtab.as<SegTab>();
    P.tab_s = c->tab_s.as<uint32_t>();
    P.tab_e = c->tab_e.as<uint32_t>();
    P.item_cap = kItemCap;
    P.rpos = c->rpos.as<uint64_t>();
    P.rcap = tot;
    P.ranges = c->ranges.as<RangeDesc>();
    P.layers = idx->d_layers;
    P.pos = idx->d_pos;
    P.sid = idx->d_sid;
    P.starts = c->starts.as<uint32_t>();
    P.ends = c->ends.as<uint32_t>();
    P.ps = c->ps.as<uint64_t>();
    P.pe = c->pe.as<uint64_t>();
    P.counts = d_counts;
    P.bp = with_bp ? d_bp : nullptr;
    P.queue = d_small + 1;
    P.rows = rows;
    P.D = D;
    P.chunk = L.chunk;
    size_t smem = (size_t)D * (with_bp ? 12 : 4);
    P.smem_tally = (rows == 1 && smem <= 160 * 1024) ? 1 : 0;
    if (!P.smem_tally) smem = 0;
    unsigned grid = (unsigned)(c->num_sms * L.ctas_per_sm);
    if (stats) RGL_CUDA(cudaEventRecord(c->ev[1], st));
    if (c->timing) RGL_TRY(timing_record(c, true));
    if (smem > 48 * 1024) {
        RGL_CUDA(cudaFuncSetAttribute(k_sweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RGL_CUDA(cudaFuncSetAttribute(k_sweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RGL_CUDA(cudaFuncSetAttribute(k_pairs<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RGL_CUDA(cudaFuncSetAttribute(k_pairs<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (with_bp) k_sweep<true><<<grid, 256, smem, st>>>(P);
    else k_sweep<false><<<grid, 256, smem, st>>>(P);
    P.queue = d_small + 2;  // the pair sweep pulls from its own counter
    if (with_bp) k_pairs<true><<<grid, 256, smem, st>>>(P);
    else k_pairs<false><<<grid, 256, smem, st>>>(P);
    launches++;
    launches++;
    RGL_CUDA(cudaGetLastError());
    if (c->timing) RGL_TRY(timing_record(c, false));
    c->last_tot = tot;
    c->last_launches = launches;
    c->last_n = n;
    if (stats) {
        RGL_CUDA(cudaEventRecord(c->ev[2], st));
        RGL_CUDA(cudaMemcpyAsync(c->h_small + 2, c->ridx.as<uint32_t>() + tot, 4, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(c->h_small + 4, d_small + 4, 8, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(c->h_small + 6, c->rpos.as<uint64_t>() + tot, 8, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(c->h_small + 8, c->ppos.as<uint64_t>() + tot, 8, cudaMemcpyDeviceToHost, st));
    }
    RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
    return RGL_OK;
}

// Maps a batch's shards to index shard ids; shards absent from the index are skipped, as the
// reference skips shards not in meta.shards (src/tasks/query/mod.rs:194-196).
int resolve_blocks(rgl_context* c, const rgl_query_batch* b, std::vector<uint32_t>* shard_ids,
                   std::vector<const rgl_query_shard*>* blocks) {
    for (uint32_t i = 0; i < b->num_shards; i++) {
        const rgl_query_shard& s = b->shards[i];
        uint32_t id;
        if (s.shard_name) {
            auto it = c->idx->shard_ids.find(s.shard_name);
            if (it == c->idx->shard_ids.end()) continue;
            id = it->second;
        } else {
            id = s.shard_id;
            if (id >= c->idx->num_shards) continue;
        }
        if (s.count == 0) continue;
        if (!s.intervals) return fail(RGL_ERR_INVALID_ARGUMENT, "query shard without intervals");
        shard_ids->push_back(id);
        blocks->push_back(&s);
    }
    return RGL_OK;
}

}  // namespace

extern "C" {

int rgl_context_create(rgl_index* index, void* stream, rgl_context** out) {
    clear_error();
    if (!index || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    auto* c = new rgl_context();
    c->idx = index;
    c->device = index->device;
    index->refs.fetch_add(1);
    int s = RGL_OK;
    if (cudaSetDevice(index->device) != cudaSuccess) s = fail(RGL_ERR_DEVICE, "cudaSetDevice");
    if (s == RGL_OK) {
        if (stream) c->stream = reinterpret_cast<cudaStream_t>(stream);
        else if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "cudaStreamCreate");
        else
            c->own_stream = true;
    }
    if (s == RGL_OK) cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, index->device);
    for (int i = 0; i < 4 && s == RGL_OK; i++)
        if (cudaEventCreate(&c->ev[i]) != cudaSuccess) s = fail(RGL_ERR_DEVICE, "cudaEventCreate");
    if (s == RGL_OK && cudaMallocHost(&c->h_small, 256) != cudaSuccess) s = fail(RGL_ERR_OOM, "pinned");
    if (s == RGL_OK) s = c->small.ensure(256);
    if (s != RGL_OK) {
        rgl_context_destroy(c);
        return s;
    }
    *out = c;
    return RGL_OK;
}

int rgl_context_destroy(rgl_context* c) {
    clear_error();
    if (!c) return RGL_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    DevBuf* bufs[] = {&c->iv, &c->blk_off, &c->blk_shard, &c->key_a, &c->key_b, &c->val_a, &c->val_b,
                      &c->ekey_a, &c->ekey_b, &c->starts, &c->ends, &c->seg, &c->segflag, &c->segnum,
                      &c->seg_begin, &c->ps_in, &c->pe_in, &c->ps, &c->pe, &c->lo, &c->hi, &c->maxhi,
                      &c->rflag, &c->ridx, &c->ranges, &c->rlen, &c->rpos, &c->cub_tmp, &c->small,
                      &c->out_counts, &c->out_bp, &c->item_r0,
                      &c->segtab, &c->tab_len, &c->tab_off, &c->tab_s, &c->tab_e,
                      &c->cl, &c->pc, &c->method, &c->ulen, &c->plen, &c->ppos, &c->psegs, &c->item_t0};
    for (DevBuf* b : bufs) b->release();
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->tev) cudaEventDestroy(e);
    if (c->h_small) cudaFreeHost(c->h_small);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    index_release(c->idx);
    delete c;
    (void)cudaGetLastError();
    return RGL_OK;
}

int rgl_context_reserve(rgl_context* c, uint64_t max_intervals, uint32_t max_rows) {
    clear_error();
    if (!c) return fail(RGL_ERR_INVALID_ARGUMENT, "null context");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    return ensure_workspace(c, max_intervals, max_rows, 4096);
}

void* rgl_context_stream(rgl_context* c) { return c ? (void*)c->stream : nullptr; }

int rgl_context_sync(rgl_context* c) {
    if (!c) return fail(RGL_ERR_INVALID_ARGUMENT, "null context");
    RGL_CUDA(cudaStreamSynchronize(c->stream));
    return RGL_OK;
}

int rgl_query_counts_device(rgl_context* c, uint32_t num_rows, uint32_t num_shards, const uint32_t* shard_ids,
                            const uint64_t* shard_offsets, const rgl_interval* d_intervals,
                            const rgl_query_opts* opts, uint32_t* d_counts, uint64_t* d_overlap_bp,
                            rgl_query_stats* stats) {
    clear_error();
    if (!c || (num_shards && (!shard_ids || !shard_offsets))) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    if (!d_counts) return fail(RGL_ERR_INVALID_ARGUMENT, "counts buffer is required");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    uint64_t n = num_shards ? shard_offsets[num_shards] - shard_offsets[0] : 0;
    if (n >= (1ull << 31)) return fail(RGL_ERR_INVALID_ARGUMENT, "at most 2^31-1 query intervals per call");
    for (uint32_t i = 0; i < num_shards; i++)
        if (shard_ids[i] >= c->idx->num_shards) return fail(RGL_ERR_INVALID_ARGUMENT, "shard id out of range");
    RGL_TRY(ensure_workspace(c, n, 0, num_shards));
    std::vector<uint64_t> off(num_shards + 1);
    for (uint32_t i = 0; i <= num_shards; i++) off[i] = shard_offsets[i] - shard_offsets[0];
    if (num_shards) {
        RGL_CUDA(cudaMemcpyAsync(c->blk_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, c->stream));
        RGL_CUDA(cudaMemcpyAsync(c->blk_shard.p, shard_ids, num_shards * 4ull, cudaMemcpyHostToDevice, c->stream));
        RGL_CUDA(cudaMemcpyAsync(c->iv.p, d_intervals + shard_offsets[0], n * sizeof(rgl_interval),
                                 cudaMemcpyDeviceToDevice, c->stream));
    }
    RGL_TRY(run_pipeline(c, n, num_rows, num_shards, opts, d_counts,
                         reinterpret_cast<unsigned long long*>(d_overlap_bp), stats));
    if (!stats) return RGL_OK;
    RGL_CUDA(cudaStreamSynchronize(c->stream));
    return finish(c, pick_launch(opts), stats);
}

int rgl_query_counts(rgl_context* c, const rgl_query_batch* b, const rgl_query_opts* opts, uint32_t* counts,
                     uint64_t* overlap_bp, rgl_query_stats* stats) {
    clear_error();
    if (!c || !b || !counts) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    std::vector<uint32_t> ids;
    std::vector<const rgl_query_shard*> blocks;
    RGL_TRY(resolve_blocks(c, b, &ids, &blocks));
    uint64_t n = 0;
    std::vector<uint64_t> off(blocks.size() + 1, 0);
    for (size_t i = 0; i < blocks.size(); i++) {
        off[i] = n;
        n += blocks[i]->count;
    }
    off[blocks.size()] = n;
    if (n >= (1ull << 31)) return fail(RGL_ERR_INVALID_ARGUMENT, "at most 2^31-1 query intervals per call");
    const uint32_t rows = b->num_rows;
    const uint64_t cells = (uint64_t)rows * c->idx->num_sources;
    RGL_TRY(ensure_workspace(c, n, rows, (uint32_t)blocks.size()));
    cudaStream_t st = c->stream;
    for (size_t i = 0; i < blocks.size(); i++)
        RGL_CUDA(cudaMemcpyAsync(c->iv.as<rgl_interval>() + off[i], blocks[i]->intervals,
                                 blocks[i]->count * sizeof(rgl_interval), cudaMemcpyHostToDevice, st));
    if (!blocks.empty()) {
        RGL_CUDA(cudaMemcpyAsync(c->blk_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st));
        RGL_CUDA(cudaMemcpyAsync(c->blk_shard.p, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, st));
    }
    RGL_TRY(run_pipeline(c, n, rows, (uint32_t)blocks.size(), opts, c->out_counts.as<uint32_t>(),
                         overlap_bp ? c->out_bp.as<unsigned long long>() : nullptr, stats));
    if (cells) {
        RGL_CUDA(cudaMemcpyAsync(counts, c->out_counts.p, cells * 4, cudaMemcpyDeviceToHost, st));
        if (overlap_bp) RGL_CUDA(cudaMemcpyAsync(overlap_bp, c->out_bp.p, cells * 8, cudaMemcpyDeviceToHost, st));
    }
    RGL_CUDA(cudaStreamSynchronize(st));
    return finish(c, pick_launch(opts), stats);
}

int rgl_context_check(rgl_context* c) {
    clear_error();
    if (!c) return fail(RGL_ERR_INVALID_ARGUMENT, "null context");
    RGL_CUDA(cudaStreamSynchronize(c->stream));
    return finish(c, pick_launch(nullptr), nullptr);
}

int rgl_context_set_timing(rgl_context* c, int on) {
    if (!c) return fail(RGL_ERR_INVALID_ARGUMENT, "null context");
    c->timing = on != 0;
    c->tev_used = 0;
    return RGL_OK;
}

int rgl_context_sweep_times(rgl_context* c, float* total_ms, uint32_t* launches) {
    if (!c || !total_ms || !launches) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    RGL_CUDA(cudaStreamSynchronize(c->stream));
    float tot = 0;
    for (size_t i = 0; i < c->tev_used; i++) {
        float ms = 0;
        RGL_CUDA(cudaEventElapsedTime(&ms, c->tev[2 * i], c->tev[2 * i + 1]));
        tot += ms;
    }
    *total_ms = tot;
    *launches = (uint32_t)c->tev_used;
    c->tev_used = 0;
    return RGL_OK;
}

int rgl_host_alloc(uint64_t bytes, void** out) {
    if (!out) return fail(RGL_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    RGL_CUDA(cudaMallocHost(out, bytes ? bytes : 1));
    return RGL_OK;
}

int rgl_host_free(void* p) {
    if (p) RGL_CUDA(cudaFreeHost(p));
    return RGL_OK;
}

}  // extern "C"
