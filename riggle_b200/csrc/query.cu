// The sweep: query_database's counting path (src/tasks/query/mod.rs:182-307) and
// query_sweep_windowed (src/sweep/query.rs:84-117) as one device pipeline.
//
// Per batch (all on the context stream, no host synchronisation, graph-capturable once the
// workspace is reserved):
//   1. k_expand_keys: each query interval becomes key (segment << 32 | start), value end, and a
//      second key (segment << 32 | end); segment = shard * rows + Q_SID.  Invalid intervals
//      (start >= end, sid >= rows) raise an error bit.
//   2. sort both key sets (the reference sorts by (sid, start), mod.rs:202; ends are sorted too,
//      which the rank formulation below needs): block by block when every input block is one
//      segment (tiles sorted in shared memory, then merge passes; ordered blocks copied through),
//      else a device-wide radix sort.
//   3. exclusive u64 prefix sums of the sorted starts and sorted ends (PS, PE).
//   4. K1 partition: for every (layer slot K, query i) the candidate range of the reference's scan,
//      [pp(start - max_K), pp(end)) with pp = partition point of the layer's starts
//      (src/sweep/query.rs:98-105); a segmented max-scan merges them into disjoint ranges per
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
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "block_sort.cuh"
#include "internal.h"

namespace rgl {

struct RangeDesc {
    uint32_t db_lo, db_hi;      // DB index range within the layer
    uint32_t c_first, c_last;   // live runs (compacted positions) whose windows formed the range
    uint32_t layer_idx;         // index into the layer table
    uint32_t qrow;              // query row (Q_SID)
    uint32_t seg;               // query segment (shard, row)
    uint32_t slot;              // layer slot K
};

// One query's candidate run for the pair sweep: DB elements [base, base + plen) of its layer.
struct PairSeg {
    uint64_t base;
    uint32_t qs, qe, qrow, shard;
};

enum : uint8_t { M_RANK = 0, M_PAIR = 1 };

// Rank table of one query segment: bin b (width 2^shift bp) holds, at tab2[off + b], the numbers
// of the segment's sorted starts and ends below b << shift, as absolute positions in the sorted
// arrays.  A rank is then one table read plus a search over at most one bin, and the two entries
// of a bin serve the start rank and the end rank of any x in it.
struct SegTab {
    uint32_t beg, end;  // the segment's positions in the sorted arrays
    uint32_t shift, nbins;
    uint32_t off;       // first entry of the segment's tables (nbins + 1 entries each)
    uint32_t pad;
};

enum : uint32_t { ERR_BAD_INTERVAL = 1u, ERR_BAD_ROW = 2u };

// Programmatic dependent launch.  The short kernels of the pipeline's chains have a PDL variant
// (template flag PDL) that starts with pdl_wait(): it returns once the grid launched before it on
// the stream has completed and its memory is visible, so nothing is read or written before it.
// pdl_release() lets the next grid of the stream be scheduled before this one finishes; that grid
// still waits in pdl_wait() for this one to complete.  Large runs launch the variants without
// either instruction.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

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
// Partition points of (start < x) over a layer sorted by start, for x0 -> r0 and x1 -> r1: the
// bucket table gives the elements whose starts share x's bucket, searched by bisection.  The two
// run in lockstep (both bucket reads issued together, then one probe of each bisection per round),
// so their chains of dependent random reads overlap instead of following one another.
__device__ __forceinline__ void pp_layer2(const uint2* __restrict__ pos, const uint32_t* __restrict__ btab,
                                          const LayerDev& L, uint32_t x0, uint32_t x1, uint32_t& r0, uint32_t& r1) {
    const uint32_t last = L.nb - 1;
    const uint32_t b0 = x0 >> L.bshift, b1 = x1 >> L.bshift;
    uint32_t lo0 = (uint32_t)L.n, hi0 = (uint32_t)L.n, lo1 = (uint32_t)L.n, hi1 = (uint32_t)L.n;
    if (b0 < last) {
        lo0 = __ldg(btab + b0);
        hi0 = __ldg(btab + b0 + 1);
    }
    if (b1 < last) {
        lo1 = __ldg(btab + b1);
        hi1 = __ldg(btab + b1 + 1);
    }
    while (lo0 < hi0 || lo1 < hi1) {
        const bool a0 = lo0 < hi0, a1 = lo1 < hi1;
        const uint32_t m0 = lo0 + ((hi0 - lo0) >> 1), m1 = lo1 + ((hi1 - lo1) >> 1);
        const uint32_t v0 = a0 ? __ldg(&pos[m0].x) : 0u, v1 = a1 ? __ldg(&pos[m1].x) : 0u;
        if (a0) {
            if (v0 < x0) lo0 = m0 + 1; else hi0 = m0;
        }
        if (a1) {
            if (v1 < x1) lo1 = m1 + 1; else hi1 = m1;
        }
    }
    r0 = lo0;
    r1 = lo1;
}

// ---- 1. keys ------------------------------------------------------------------------------------
__global__ void k_expand_keys(uint32_t n, const rgl_interval* __restrict__ iv, const uint64_t* __restrict__ blk_off,
                              const uint32_t* __restrict__ blk_shard, const uint32_t* __restrict__ blk_row,
                              int row_from_block, uint32_t nblk, uint32_t rows, uint32_t row_base, uint32_t rb,
                              uint64_t* __restrict__ key, uint32_t* __restrict__ val, uint64_t* __restrict__ ekey,
                              uint32_t* __restrict__ err, uint32_t* __restrict__ unsorted,
                              const uint64_t* __restrict__ sdst, const uint32_t* __restrict__ sidx) {
    // block b with blk_off[b] <= i < blk_off[b+1]: one search per thread block, for its first
    // element, then a short walk (256 consecutive elements span few blocks)
    __shared__ uint32_t s_b0;
    const uint32_t i0 = blockIdx.x * blockDim.x, i = i0 + threadIdx.x;
    if (threadIdx.x == 0) {
        uint32_t lo = 0, hi = nblk;
        while (hi - lo > 1) {
            const uint32_t m = (lo + hi) >> 1;
            if (blk_off[m] <= i0) lo = m; else hi = m;
        }
        s_b0 = lo;
    }
    __syncthreads();
    if (i >= n) return;
    uint32_t lo = s_b0;
    while (lo + 1 < nblk && blk_off[lo + 1] <= i) lo++;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(iv) + 3ull * i;
    // the block-local sort: block b's keys at sdst[b] + their place in the block (segment-order
    // layout) or in place; order flags of the block's rank k in that layout: starts (ends) out of
    // order -> unsorted[k] (unsorted[nblk + k]) = 1
    const uint64_t o = sdst ? sdst[lo] + (i - blk_off[lo]) : (uint64_t)i;
    if (unsorted && i > blk_off[lo]) {
        const uint32_t k = sidx ? sidx[lo] : lo;
        if (w[0] < w[-3]) unsorted[k] = 1u;
        if (w[1] < w[-2]) unsorted[nblk + k] = 1u;
    }
    // the row is the interval's sid, or with row_from_block its block's row (sid ignored)
    const uint32_t row = row_from_block ? blk_row[lo] : w[2];
    uint32_t s = w[0], e = w[1], q = row - row_base;  // rows below row_base wrap to >= rows
    uint32_t bad = 0;
    if (s >= e) bad |= ERR_BAD_INTERVAL;
    if (q >= rows || (blk_row && row != blk_row[lo])) { bad |= ERR_BAD_ROW; q = 0; }
    if (bad) atomicOr(err, bad);
    // segment = (shard, region, row): with regions (rb > 0) a row's intervals on a shard are cut
    // into 2^rb-bp regions of their starts, so that the rows' work on one region lies together
    const uint64_t nreg = rb ? (1ull << (32 - rb)) : 1ull, reg = rb ? (s >> rb) : 0u;
    uint64_t seg = ((uint64_t)blk_shard[lo] * nreg + reg) * rows + q;
    key[o] = (seg << 32) | s;
    val[o] = e;
    ekey[o] = (seg << 32) | e;
}

// The sorted start keys into starts, segment ids, segment-start flags and the starts' prefix-sum
// input (entry n = 0); the sorted end keys into ends and the ends' prefix-sum input.
__global__ void k_unpack_starts(uint32_t n, const uint64_t* __restrict__ key, uint32_t* __restrict__ starts,
                                uint32_t* __restrict__ seg, uint32_t* __restrict__ segflag,
                                uint64_t* __restrict__ ps_in) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        ps_in[n] = 0;
        return;
    }
    const uint64_t k = key[i];
    const uint32_t s = (uint32_t)k, sg = (uint32_t)(k >> 32);
    starts[i] = s;
    seg[i] = sg;
    segflag[i] = (i == 0 || (uint32_t)(key[i - 1] >> 32) != sg) ? 1u : 0u;
    ps_in[i] = s;
}
__global__ void k_unpack_ends(uint32_t n, const uint64_t* __restrict__ ekey, uint32_t* __restrict__ ends_s,
                              uint64_t* __restrict__ pe_in) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        pe_in[n] = 0;
        return;
    }
    const uint32_t e = (uint32_t)ekey[i];
    ends_s[i] = e;
    pe_in[i] = e;
}

__global__ void k_seg_begin(uint32_t n, const uint32_t* __restrict__ segflag, const uint32_t* __restrict__ segnum,
                            uint32_t* __restrict__ seg_begin) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (segflag[i]) seg_begin[segnum[i] - 1] = i;
    if (i == n - 1) seg_begin[segnum[i]] = n;
}

// Bin width per segment: about four bins per query, at least 64 bp, but no more than one bin per 8
// DB intervals the segment's rank-difference ranges sweep (need[]): each swept interval reads the
// table a few times, so a table much larger than its sweep costs more to build than its finer bins
// save (large query files against a small database).  A coarser bin only lengthens the search
// inside it.  A segment with a rank-difference range gets nbins + 1 table entries, any other
// segment a single entry (see k_tab_place).
__global__ void k_seg_tabsize(uint32_t n, const uint32_t* __restrict__ segnum, const uint32_t* __restrict__ seg_begin,
                              const unsigned long long* __restrict__ need, const uint32_t* __restrict__ ends_s,
                              SegTab* __restrict__ tabs, uint32_t* __restrict__ tab_len) {
    uint32_t sgi = blockIdx.x * blockDim.x + threadIdx.x;
    if (sgi > n) return;
    const uint32_t nseg = segnum[n - 1];
    if (sgi >= nseg) {
        tab_len[sgi] = 0;
        return;
    }
    const uint32_t beg = seg_begin[sgi], end = seg_begin[sgi + 1];
    if (!need[sgi]) {  // no range of this segment is swept by rank differences
        tabs[sgi] = SegTab{beg, end, 6, 0, 0, 0};
        tab_len[sgi] = 1;
        return;
    }
    const uint64_t extent = (uint64_t)ends_s[end - 1] + 1;  // covers every start and end of the segment
    const uint64_t bins = max(1ull, min(4ull * (end - beg), need[sgi] / 8));
    const uint64_t want = extent / bins;
    uint32_t shift = want > 1 ? 63u - __clzll(want) : 0u;
    if (shift < 6) shift = 6;
    if (shift > 31) shift = 31;
    const uint32_t nbins = (uint32_t)(extent >> shift) + 1;  // <= 8 (end - beg): tables fit 10 n entries
    tabs[sgi] = SegTab{beg, end, shift, nbins, 0, 0};
    tab_len[sgi] = nbins + 1;
}

// Rank tables by counting.  Entry b of a segment's table must hold beg + #{elements with bin < b}.
// With the per-bin counts placed one entry to the right (bin b at entry b + 1) and every other
// segment's single entry holding its element count, an inclusive scan over all segments' entries
// yields exactly that: everything before a segment's first entry sums to its `beg`.
// Zeroes the count arrays over the tables' actual size (tab_off[number of segments]) and records
// that size in *count for the scans.
__global__ void k_tab_zero(uint32_t n, const uint32_t* __restrict__ segnum, const uint32_t* __restrict__ tab_off,
                           uint32_t* __restrict__ xs, uint32_t* __restrict__ xe, uint32_t* __restrict__ count) {
    const uint32_t total = tab_off[segnum[n - 1]];
    const uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (g == 0) *count = total;
    for (uint64_t i = g; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        xs[i] = 0;
        xe[i] = 0;
    }
}

template <bool PDL>
__global__ void k_tab_place(uint32_t n, const uint32_t* __restrict__ segnum, SegTab* __restrict__ tabs,
                            const uint32_t* __restrict__ tab_off, uint32_t* __restrict__ xs, uint32_t* __restrict__ xe) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t sgi = blockIdx.x * blockDim.x + threadIdx.x;
    if (sgi >= segnum[n - 1]) return;
    const uint32_t off = tab_off[sgi];
    tabs[sgi].off = off;
    const SegTab t = tabs[sgi];
    if (t.nbins == 0) {
        xs[off] = t.end - t.beg;
        xe[off] = t.end - t.beg;
    }
}

template <bool PDL>
__global__ void k_tab_count(uint32_t n, const uint32_t* __restrict__ segnum, const SegTab* __restrict__ tabs,
                            const uint32_t* __restrict__ starts, const uint32_t* __restrict__ ends_s,
                            uint32_t* __restrict__ xs, uint32_t* __restrict__ xe) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const SegTab t = tabs[segnum[j] - 1];
    if (t.nbins == 0) return;
    atomicAdd(xs + t.off + (starts[j] >> t.shift) + 1, 1u);
    atomicAdd(xe + t.off + (ends_s[j] >> t.shift) + 1, 1u);
}

// Adds a 32-bit value to a 64-bit shared-memory counter with 32-bit atomics: the low word, and the
// high word only when the low word wraps (one pair's overlap always fits 32 bits).
__device__ __forceinline__ void add_u64_lo(unsigned long long* c, uint32_t v) {
    uint32_t* w = reinterpret_cast<uint32_t*>(c);  // little-endian: w[0] low, w[1] high
    const uint32_t old = atomicAdd(w, v);
    if (old + v < old) atomicAdd(w + 1, 1u);
}

// The same for a 64-bit value: low word, then the high word plus the carry when either is non-zero.
__device__ __forceinline__ void add_u64(unsigned long long* c, unsigned long long v) {
    uint32_t* w = reinterpret_cast<uint32_t*>(c);
    const uint32_t lo = (uint32_t)v, old = atomicAdd(w, lo);
    const uint32_t hi = (uint32_t)(v >> 32) + (old + lo < old ? 1u : 0u);
    if (hi) atomicAdd(w + 1, hi);
}

// Interleaves the two scanned count arrays into (#starts, #ends) pairs: entry k of the tables is
// entry k + 1 of the exclusive scans (the inclusive sums through k).
template <bool PDL>
__global__ void k_tab_interleave(const uint32_t* __restrict__ count, const uint32_t* __restrict__ xs_scan,
                                 const uint32_t* __restrict__ xe_scan, uint2* __restrict__ tab2) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t total = *count;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x)
        tab2[k] = make_uint2(xs_scan[k + 1], xe_scan[k + 1]);
}

// ---- 4. K1 partition -----------------------------------------------------------------------------
// lo/hi of the reference's candidate scan for (slot K, query i), layer-major arrays [K][n].
__global__ void k_lohi(uint32_t n, uint32_t nslots, uint32_t seg_per_shard, const uint32_t* __restrict__ starts,
                       const uint32_t* __restrict__ qend, const uint32_t* __restrict__ seg,
                       const int32_t* __restrict__ slot, const LayerDev* __restrict__ layers,
                       const uint2* __restrict__ pos, const uint32_t* __restrict__ btab,
                       uint32_t* __restrict__ lo_out, uint32_t* __restrict__ hi_out, uint32_t* __restrict__ live) {
    // grid: x over the queries, y over the layer slots (no 64-bit division per thread)
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, K = blockIdx.y;
    if (i >= n) return;
    const uint64_t t = (uint64_t)K * n + i;
    uint32_t shard = seg[i] / seg_per_shard;
    int32_t li = slot[(uint64_t)shard * nslots + K];
    uint32_t lo = 0, hi = 0;
    if (li >= 0) {
        LayerDev L = layers[li];
        const uint2* p = pos + L.off;
        uint32_t s = starts[i];
        uint32_t back = s >= L.max_size ? s - L.max_size : 0u;  // saturating_sub, src/sweep/query.rs:98
        const uint32_t* bt = btab + L.boff;
        pp_layer2(p, bt, L, back, qend[i], lo, hi);
        if (hi < lo) hi = lo;
    }
    lo_out[t] = lo;
    hi_out[t] = hi;
    // the live-run flags of the compaction below (entry n * nslots: the scan's closing zero)
    live[t] = hi > lo ? 1u : 0u;
    if (t == 0) live[(uint64_t)n * nslots] = 0u;
}

// ---- scans whose length is a device count ------------------------------------------------------
// After the compaction below, the number of entries (live candidate runs, ranges) is known only on
// the device; these scans read it there, so the pipeline keeps no host synchronisation (and stays
// graph-capturable) while its work follows the live count instead of the (query, slot) capacity.
// Exclusive scan of in[0, n) into out[0, n], out[n] = total: per-tile sums, one block scanning the
// tile sums, per-tile block scans offset by them.  The tile kernels are launched with a grid sized
// for the SMs and walk the tiles below n grid-stride, so a capacity far above the live count costs
// no empty blocks.
constexpr int kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

template <typename Tin, typename Tout, bool PDL>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const Tin* __restrict__ in,
                                                              const uint32_t* __restrict__ n_ptr,
                                                              Tout* __restrict__ tile_sums) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t n = *n_ptr;
    using BR = cub::BlockReduce<Tout, kScanThreads>;
    __shared__ typename BR::TempStorage tmp;
    for (uint64_t tile = blockIdx.x; tile * kScanTile < n; tile += gridDim.x) {
        const uint64_t base = tile * kScanTile;
        Tout s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            const uint64_t i = base + (uint64_t)k * kScanThreads + threadIdx.x;
            if (i < n) s += (Tout)in[i];
        }
        s = BR(tmp).Sum(s);
        if (threadIdx.x == 0) tile_sums[tile] = s;
        __syncthreads();  // tmp is reused by the next tile
    }
}

template <typename Tout, bool PDL>
__global__ void __launch_bounds__(1024) k_scan_tops(Tout* __restrict__ tile_sums, const uint32_t* __restrict__ n_ptr,
                                                    Tout* __restrict__ out) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t n = *n_ptr;
    const uint32_t nt = (uint32_t)((n + kScanTile - 1) / kScanTile);
    using BS = cub::BlockScan<Tout, 1024>;
    __shared__ typename BS::TempStorage tmp;
    Tout run = 0;
    for (uint32_t b0 = 0; b0 < nt; b0 += 1024) {
        const uint32_t b = b0 + threadIdx.x;
        Tout v = b < nt ? tile_sums[b] : (Tout)0, ex, agg;
        BS(tmp).ExclusiveSum(v, ex, agg);
        if (b < nt) tile_sums[b] = run + ex;
        run += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = run;
}

template <typename Tin, typename Tout, bool PDL>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const Tin* __restrict__ in, Tout* __restrict__ out,
                                                             const uint32_t* __restrict__ n_ptr,
                                                             const Tout* __restrict__ tile_off) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t n = *n_ptr;
    using BL = cub::BlockLoad<Tout, kScanThreads, kScanItems, cub::BLOCK_LOAD_WARP_TRANSPOSE>;
    using BSt = cub::BlockStore<Tout, kScanThreads, kScanItems, cub::BLOCK_STORE_WARP_TRANSPOSE>;
    using BS = cub::BlockScan<Tout, kScanThreads>;
    __shared__ union {
        typename BL::TempStorage load;
        typename BSt::TempStorage store;
        typename BS::TempStorage scan;
    } tmp;
    for (uint64_t tile = blockIdx.x; tile * kScanTile < n; tile += gridDim.x) {
        const uint64_t base = tile * kScanTile;
        const int valid = (int)((uint64_t)n - base < (uint64_t)kScanTile ? (uint64_t)n - base : (uint64_t)kScanTile);
        Tout v[kScanItems];
        BL(tmp.load).Load(in + base, v, valid, (Tout)0);
        __syncthreads();
        BS(tmp.scan).ExclusiveSum(v, v);
        const Tout off = tile_off[tile];
#pragma unroll
        for (int k = 0; k < kScanItems; k++) v[k] += off;
        __syncthreads();
        BSt(tmp.store).Store(out + base, v, valid);
        __syncthreads();  // tmp is reused by the next tile
    }
}

// ---- running maximum of hi over the live runs of each (slot, segment) row -----------------------
// maxc[c] = max of hi over the live entries of entry c's row up to c.  Empty entries never raise the
// running maximum past a later entry's lo (see 4b), so the maximum over live entries alone decides
// every range exactly as the maximum over all entries would.  A segmented scan over the L live
// entries (a device count): per-tile summaries (head seen, maximum since the last head), one block
// scanning them into each tile's carry, per-tile block scans with the carry.
struct SegMax {
    uint32_t f, v;  // f: the span holds a row start; v: maximum since the span's last row start
};
struct SegMaxOp {
    __device__ __forceinline__ SegMax operator()(const SegMax& a, const SegMax& b) const {
        return SegMax{a.f | b.f, b.f ? b.v : max(a.v, b.v)};
    }
};

// Live entry c as a scan item: its hi and whether it starts a (slot, segment) row.
__device__ __forceinline__ SegMax segmax_item(uint64_t c, const uint32_t* __restrict__ tl, uint32_t n,
                                              const uint32_t* __restrict__ segnum, const uint32_t* __restrict__ hi) {
    const uint32_t t = tl[c];
    bool head = c == 0;
    if (!head) {
        const uint32_t tp = tl[c - 1];
        head = (tp / n != t / n) || (segnum[tp % n] != segnum[t % n]);
    }
    return SegMax{head ? 1u : 0u, hi[t]};
}

template <bool PDL>
__global__ void __launch_bounds__(kScanThreads) k_segmax_reduce(const uint32_t* __restrict__ Lp, uint32_t n,
                                                                const uint32_t* __restrict__ tl,
                                                                const uint32_t* __restrict__ segnum,
                                                                const uint32_t* __restrict__ hi,
                                                                unsigned long long* __restrict__ tile_sums) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t L = *Lp;
    using BS = cub::BlockScan<SegMax, kScanThreads>;
    __shared__ typename BS::TempStorage tmp;
    for (uint64_t tile = blockIdx.x; tile * kScanTile < L; tile += gridDim.x) {
        const uint64_t base = tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
        SegMax v[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; k++)
            v[k] = base + k < L ? segmax_item(base + k, tl, n, segnum, hi) : SegMax{0u, 0u};
        SegMax agg;
        BS(tmp).InclusiveScan(v, v, SegMaxOp(), agg);
        if (threadIdx.x == 0) tile_sums[tile] = ((unsigned long long)agg.f << 32) | agg.v;
        __syncthreads();  // tmp is reused by the next tile
    }
}

// tile_sums[t] <- the running maximum carried into tile t (the value before its first row start).
template <bool PDL>
__global__ void __launch_bounds__(1024) k_segmax_tops(const uint32_t* __restrict__ Lp,
                                                      unsigned long long* __restrict__ tile_sums) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t L = *Lp;
    const uint32_t nt = (uint32_t)((L + kScanTile - 1) / kScanTile);
    using BS = cub::BlockScan<SegMax, 1024>;
    __shared__ typename BS::TempStorage tmp;
    SegMax run{0u, 0u};
    for (uint32_t b0 = 0; b0 < nt; b0 += 1024) {
        const uint32_t b = b0 + threadIdx.x;
        const unsigned long long w = b < nt ? tile_sums[b] : 0ull;
        SegMax v{(uint32_t)(w >> 32), (uint32_t)w}, ex, agg;
        BS(tmp).ExclusiveScan(v, ex, SegMax{0u, 0u}, SegMaxOp(), agg);
        const SegMax carry = threadIdx.x ? SegMaxOp()(run, ex) : run;
        __syncthreads();  // every thread has read its summary before any is overwritten
        if (b < nt) tile_sums[b] = carry.v;
        run = SegMaxOp()(run, agg);
        __syncthreads();
    }
}

template <bool PDL>
__global__ void __launch_bounds__(kScanThreads) k_segmax_apply(const uint32_t* __restrict__ Lp, uint32_t n,
                                                               const uint32_t* __restrict__ tl,
                                                               const uint32_t* __restrict__ segnum,
                                                               const uint32_t* __restrict__ hi,
                                                               const unsigned long long* __restrict__ carry,
                                                               uint32_t* __restrict__ maxc) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t L = *Lp;
    using BS = cub::BlockScan<SegMax, kScanThreads>;
    __shared__ typename BS::TempStorage tmp;
    for (uint64_t tile = blockIdx.x; tile * kScanTile < L; tile += gridDim.x) {
        const uint64_t base = tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
        SegMax v[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; k++)
            v[k] = base + k < L ? segmax_item(base + k, tl, n, segnum, hi) : SegMax{0u, 0u};
        if (threadIdx.x == 0 && !v[0].f) v[0].v = max(v[0].v, (uint32_t)carry[tile]);
        BS(tmp).InclusiveScan(v, v, SegMaxOp());
#pragma unroll
        for (int k = 0; k < kScanItems; k++)
            if (base + k < L) maxc[base + k] = v[k].v;
        __syncthreads();  // tmp is reused by the next tile
    }
}

// ---- 4b. live candidate runs -------------------------------------------------------------------
// An entry (K, i) whose run [lo, hi) is empty takes part in nothing: with starts sorted, lo is
// non-decreasing within a (K, segment) row, so an empty run's hi (= its lo) never exceeds a later
// entry's lo and can neither merge nor split ranges.  The live entries are compacted (tl[c] = t,
// c < L, by a flagged selection) and everything after this works on them.  k_lohi writes the live
// flags with lo and hi.

// Range starts among the live runs: the first live run of a (K, segment) row, or one whose lo is
// past the running maximum of hi over the row's earlier live runs (maxhi[c - 1]); cl = the run's
// candidate count.
template <bool PDL>
__global__ void k_crange_flags(const uint32_t* __restrict__ Lp, uint32_t n, const uint32_t* __restrict__ tl,
                               const uint32_t* __restrict__ segnum, const uint32_t* __restrict__ lo,
                               const uint32_t* __restrict__ hi, const uint32_t* __restrict__ maxhi,
                               uint32_t* __restrict__ cflag, uint64_t* __restrict__ ccl) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t L = *Lp;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < L; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = tl[c];
        bool start = c == 0;
        if (!start) {
            const uint32_t tp = tl[c - 1];
            start = (tp / n != t / n) || (segnum[tp % n] != segnum[t % n]) || (lo[t] >= maxhi[c - 1]);
        }
        cflag[c] = start ? 1u : 0u;
        ccl[c] = (uint64_t)(hi[t] - lo[t]);
    }
}

template <bool PDL>
__global__ void k_crange_emit(const uint32_t* __restrict__ Lp, uint32_t n, uint32_t nslots, uint32_t rows,
                              uint32_t seg_per_shard, const uint32_t* __restrict__ tl, const uint32_t* __restrict__ seg,
                              const uint32_t* __restrict__ segnum, const int32_t* __restrict__ slot,
                              const uint32_t* __restrict__ lo, const uint32_t* __restrict__ maxhi,
                              const uint32_t* __restrict__ cflag, const uint32_t* __restrict__ cridx,
                              RangeDesc* __restrict__ ranges) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t L = *Lp;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < L; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = tl[c], K = t / n, i = t % n;
        const uint32_t f = cflag[c];
        const uint32_t r = cridx[c] + f - 1;  // inclusive range index
        if (f) {
            const uint32_t sg = seg[i];
            ranges[r].db_lo = lo[t];
            ranges[r].c_first = (uint32_t)c;
            ranges[r].layer_idx = (uint32_t)slot[(uint64_t)(sg / seg_per_shard) * nslots + K];
            ranges[r].qrow = sg % rows;
            ranges[r].seg = segnum[i] - 1;
            ranges[r].slot = K;
        }
        if (c + 1 == L || cflag[c + 1]) {
            ranges[r].c_last = (uint32_t)c;
            ranges[r].db_hi = maxhi[c];
        }
    }
}

// Per range: the reference's candidate count (sum over its runs of hi - lo) against the size of the
// union.  Where the two are close (narrow layers) the pair sweep reads each candidate once with
// trivial per-pair work; where candidate windows overlap heavily (broad layers) the rank sweep reads
// each union element once.  rlen = union length of rank ranges (the rank work space); the union of
// every range is summed into *union_total (the swept count of the metric).
template <bool PDL>
__global__ void __launch_bounds__(256) k_crange_method(const uint32_t* __restrict__ Lp, const uint32_t* __restrict__ cridx,
                                const RangeDesc* __restrict__ ranges, const uint64_t* __restrict__ cpc,
                                uint32_t pair_ratio, uint8_t* __restrict__ method, uint64_t* __restrict__ rlen,
                                unsigned long long* __restrict__ seg_need, uint32_t* __restrict__ R_out,
                                unsigned long long* __restrict__ union_total) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t R = cridx[*Lp];
    const uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (g == 0) *R_out = R;
    unsigned long long acc = 0;
    for (uint64_t r = g; r < R; r += (uint64_t)gridDim.x * blockDim.x) {
        const RangeDesc rd = ranges[r];
        const uint64_t len = rd.db_hi - rd.db_lo;
        const uint64_t cand = cpc[rd.c_last + 1] - cpc[rd.c_first];
        const uint8_t m = (cand <= (uint64_t)pair_ratio * len) ? M_PAIR : M_RANK;
        method[r] = m;
        if (m == M_RANK && len) atomicAdd(&seg_need[rd.seg], (unsigned long long)len);  // rank-swept positions
        rlen[r] = m == M_RANK ? len : 0;
        acc += len;
    }
    // one atomic per block on the shared total
    using BR = cub::BlockReduce<unsigned long long, 256>;
    __shared__ typename BR::TempStorage tmp;
    acc = BR(tmp).Sum(acc);
    if (threadIdx.x == 0 && acc) atomicAdd(union_total, acc);
}

// Pair work space: each live run of a pair range contributes its candidates.
template <bool PDL>
__global__ void k_cpair_len(const uint32_t* __restrict__ Lp, uint32_t n, uint32_t nslots, uint32_t rows,
                            uint32_t seg_per_shard, const uint32_t* __restrict__ tl, const uint32_t* __restrict__ seg,
                            const int32_t* __restrict__ slot, const LayerDev* __restrict__ layers,
                            const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi,
                            const uint32_t* __restrict__ cflag, const uint32_t* __restrict__ cridx,
                            const uint8_t* __restrict__ method, const uint32_t* __restrict__ starts,
                            const uint32_t* __restrict__ qend, uint64_t* __restrict__ plen,
                            PairSeg* __restrict__ psegs) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t L = *Lp;
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < L; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = tl[c], K = t / n, i = t % n;
        const uint32_t r = cridx[c] + cflag[c] - 1;
        uint64_t len = 0;
        if (method[r] == M_PAIR) {
            const uint32_t sg = seg[i];
            const int32_t li = slot[(uint64_t)(sg / seg_per_shard) * nslots + K];
            len = hi[t] - lo[t];
            psegs[c] = PairSeg{layers[li].off + lo[t], starts[i], qend[i], sg % rows, sg / seg_per_shard};
        }
        plen[c] = len;
    }
}

// Totals of the rank and pair work spaces (stats): small[10..11] = rpos[R], small[12..13] = ppos[L].
__global__ void k_totals(uint32_t* __restrict__ small, const uint64_t* __restrict__ rpos,
                         const uint64_t* __restrict__ ppos) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned long long* s64 = reinterpret_cast<unsigned long long*>(small);
        s64[5] = rpos[small[9]];
        s64[6] = ppos[small[8]];
    }
}

struct SweepParams {
    const uint64_t* rpos;   // exclusive scan of rank-range lengths, R + 1 entries; rpos[R] = total
    const uint32_t* rcount; // R (device): ranges
    const uint32_t* pcount; // L (device): live candidate runs
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
    const uint64_t* ppos;    // pair work space: exclusive scan of candidate runs, L + 1 entries
    const PairSeg* psegs;
    const uint32_t* item_t0; // first run of each pair work item
    const SegTab* segtabs;   // per query segment
    const uint2* tab2;       // rank tables, bin b = (#starts, #ends) below b << shift
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
// found by binary search over the range offsets.  One launch serves the rank ranges (rpos, *Rp
// ranges) and the pair runs (ppos, *Lp runs), grid-stride over the items of both, and records the
// two position totals in the counter block (64-bit words 5 and 6).
template <bool PDL>
__global__ void k_item_ranges(uint32_t* __restrict__ small, const uint32_t* __restrict__ Rp,
                              const uint64_t* __restrict__ rpos, const uint32_t* __restrict__ Lp,
                              const uint64_t* __restrict__ ppos, uint32_t chunk, uint64_t item_cap,
                              uint32_t* __restrict__ item_r0, uint32_t* __restrict__ item_t0) {
    if constexpr (PDL) {
        pdl_wait();
        pdl_release();
    }
    const uint32_t R = *Rp, L = *Lp;
    const uint64_t rtot = rpos[R], ptot = ppos[L];
    const uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (g0 == 0) {
        unsigned long long* s64 = reinterpret_cast<unsigned long long*>(small);
        s64[5] = rtot;
        s64[6] = ptot;
    }
    const uint64_t ri = min((rtot + chunk - 1) / chunk, item_cap);
    const uint64_t pi = min((ptot + chunk - 1) / chunk, item_cap);
    for (uint64_t g = g0; g < ri + pi; g += (uint64_t)gridDim.x * blockDim.x) {
        const bool rank = g < ri;
        const uint64_t* a = rank ? rpos : ppos;
        const uint64_t i = rank ? g : g - ri;
        const uint64_t p = i * chunk;
        uint64_t lo = 0, hi = rank ? R : L;
        while (lo < hi) {
            uint64_t m = (lo + hi + 1) >> 1;
            if (__ldg(a + m) <= p) lo = m; else hi = m - 1;
        }
        (rank ? item_r0 : item_t0)[i] = (uint32_t)lo;
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

__device__ __forceinline__ void cursor_seek(const SweepParams& P, Cursor& c, uint64_t p, uint32_t rcap) {
    if (p >= c.rhi) cursor_load(P, c, range_advance(P.rpos, c.r, rcap, p));
}

// Bin entries (#starts, #ends) b and b + 1 for the bin of x, or (end, end) twice past the table.
__device__ __forceinline__ void bin_pair(const SweepParams& P, const SegTab& t, uint32_t x, uint2& lo, uint2& hi) {
    const uint32_t b = x >> t.shift;
    if (b >= t.nbins) {
        lo = hi = make_uint2(t.end, t.end);
        return;
    }
    lo = __ldg(P.tab2 + t.off + b);
    hi = __ldg(P.tab2 + t.off + b + 1);
}
// Ranks inside one bin: #starts < x given the bin's start counts, #ends <= x given its end counts.
__device__ __forceinline__ uint32_t starts_in(const SweepParams& P, uint32_t lo, uint32_t hi, uint32_t x) {
    return lo == hi ? lo : lb_u32(P.starts, lo, hi, x);
}
__device__ __forceinline__ uint32_t ends_in(const SweepParams& P, uint32_t lo, uint32_t hi, uint32_t x) {
    return lo == hi ? lo : ub_u32(P.ends, lo, hi, x);
}

// One DB interval d with the table entries of its start's bin (a0, a1) and its end's bin (b0, b1):
// count(d) = #{q.start < d.end} - #{q.end <= d.start}, and for a non-zero count the overlap
// Cov(d.end) - Cov(d.start) and the tally.
template <bool WITH_BP, bool MULTI>
__device__ __forceinline__ void sweep_one(const SweepParams& P, uint32_t qrow, uint2 d, uint32_t sid, uint2 a0,
                                          uint2 a1, uint2 b0, uint2 b1, uint32_t* s_cnt,
                                          unsigned long long* s_bp, uint32_t cta_row) {
    const uint32_t el_s = ends_in(P, a0.y, a1.y, d.x);
    const uint32_t sl_e = starts_in(P, b0.x, b1.x, d.y);
    const uint32_t cnt = sl_e - el_s;
    if (!cnt) return;
    unsigned long long bpv = 0;
    if (WITH_BP) {
        const uint32_t sl_s = starts_in(P, a0.x, a1.x, d.x);
        const uint32_t el_e = ends_in(P, b0.y, b1.y, d.y);
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
    // one-row runs tally in the block's histogram; several-row runs (MULTI) in the histogram of the
    // block's current row, and only the other rows in the output matrix
    if (MULTI ? qrow == cta_row : P.smem_tally != 0) {
        atomicAdd(&s_cnt[sid], cnt);
        if (WITH_BP) add_u64(&s_bp[sid], bpv);
    } else {
        const uint64_t cell = (uint64_t)qrow * P.D + sid;
        atomicAdd(&P.counts[cell], cnt);
        if (WITH_BP) atomicAdd(&P.bp[cell], bpv);
    }
}

// Work items of the several-row sweeps are pulled by whole blocks: block item ci is the kCtaItems
// warp items [ci * kCtaItems, (ci + 1) * kCtaItems), one per warp.
constexpr uint32_t kCtaItems = 8;  // warps of a 256-thread block

// The row of the middle of block item ci (its warp item ci * kCtaItems + kCtaItems / 2, or the last
// item), from the first range (RANK) or run of that warp item: the row the block's histogram serves.
template <bool RANK>
__device__ __forceinline__ uint32_t cta_item_row(const SweepParams& P, uint64_t ci, uint64_t items, uint32_t rcap) {
    const uint64_t wi = min(ci * kCtaItems + kCtaItems / 2, items - 1);
    const uint64_t* off = RANK ? P.rpos : P.ppos;
    uint32_t r;
    if (wi < P.item_cap) {
        r = __ldg((RANK ? P.item_r0 : P.item_t0) + wi);
    } else {
        const uint64_t p = wi * P.chunk;
        uint64_t lo = 0, hi = rcap;
        while (lo < hi) { uint64_t m = (lo + hi + 1) >> 1; if (__ldg(off + m) <= p) lo = m; else hi = m - 1; }
        r = (uint32_t)lo;
    }
    return RANK ? P.ranges[r].qrow : P.psegs[r].qrow;
}

// The outer loop of the several-row sweeps.  Blocks pull block items (kCtaItems warp items) from the
// queue one at a time, so that the blocks running at once work on neighbouring items: with the
// region work order they read the same database region, from L2 after the first.  The block's
// histogram serves one row at a time: before an item whose row differs from the row it holds, it is
// added to the outputs and cleared (and once more at the end).  item_fn(warp_item, row) walks one
// warp item; flush_fn(row) adds and clears the histogram.
template <bool RANK, typename ItemFn, typename FlushFn>
__device__ __forceinline__ void multi_row_loop(const SweepParams& P, uint64_t items, uint32_t rcap, ItemFn item_fn,
                                               FlushFn flush_fn) {
    __shared__ uint32_t s_ctl[2];
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    uint32_t cur = kNone;  // the row the histogram holds (block-uniform)
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t ci = atomicAdd(P.queue, 1u);
            s_ctl[0] = ci;
            if ((uint64_t)ci * kCtaItems < items) s_ctl[1] = cta_item_row<RANK>(P, ci, items, rcap);
        }
        __syncthreads();
        const uint64_t ci = s_ctl[0];
        const uint32_t row = s_ctl[1];
        __syncthreads();  // every thread has read s_ctl
        if (ci * kCtaItems >= items) break;
        if (row != cur) {
            if (cur != kNone) {
                flush_fn(cur);
                __syncthreads();
            }
            cur = row;
        }
        const uint64_t item = ci * kCtaItems + (threadIdx.x >> 5);
        if (item < items) item_fn((uint32_t)item, cur);
        __syncthreads();  // the item is done before the histogram may be flushed
    }
    if (cur != kNone) flush_fn(cur);
}

// Adds the block's histogram to row `row` of the outputs and clears it (between two __syncthreads).
template <bool WITH_BP>
__device__ __forceinline__ void flush_row(const SweepParams& P, uint32_t row, uint32_t* s_cnt,
                                          unsigned long long* s_bp) {
    const uint64_t base = (uint64_t)row * P.D;
    for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
        const uint32_t c = s_cnt[k];
        if (c) {
            atomicAdd(&P.counts[base + k], c);
            s_cnt[k] = 0;
        }
        if (WITH_BP) {
            const unsigned long long b = s_bp[k];
            if (b) {
                atomicAdd(&P.bp[base + k], b);
                s_bp[k] = 0;
            }
        }
    }
}

constexpr uint32_t kUnroll = 2;      // DB intervals per lane per step of the rank sweep
constexpr uint32_t kPairUnroll = 4;  // candidates per lane per step of the pair sweep

// One work item of the rank sweep: positions [item * chunk, (item + 1) * chunk) of the concatenated
// rank ranges, walked by one warp.
template <bool WITH_BP, bool MULTI>
__device__ __forceinline__ void sweep_item(const SweepParams& P, uint32_t item, uint32_t lane, uint32_t rcap,
                                           uint64_t total, uint32_t* s_cnt, unsigned long long* s_bp,
                                           uint32_t cta_row) {
    const uint64_t p0 = (uint64_t)item * P.chunk;
    const uint64_t p1 = min(p0 + P.chunk, total);
    uint32_t r0;
    if (item < P.item_cap) {
        r0 = __ldg(P.item_r0 + item);
    } else {
        uint64_t lo = 0, hi = rcap;
        while (lo < hi) { uint64_t m = (lo + hi + 1) >> 1; if (__ldg(P.rpos + m) <= p0) lo = m; else hi = m - 1; }
        r0 = (uint32_t)lo;
    }
    Cursor c;
    cursor_load(P, c, r0);
    for (uint64_t pb = p0 + lane; pb < p1; pb += 32 * kUnroll) {
        const uint64_t plast = min(pb + 32 * (kUnroll - 1), p1 - 1 - ((p1 - 1 - pb) & 31));
        cursor_seek(P, c, pb, rcap);
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
            uint2 a0[kUnroll], a1[kUnroll], b0[kUnroll], b1[kUnroll];
#pragma unroll
            for (uint32_t j = 0; j < kUnroll; j++) {
                bin_pair(P, t, d[j].x, a0[j], a1[j]);
                bin_pair(P, t, d[j].y, b0[j], b1[j]);
            }
#pragma unroll
            for (uint32_t j = 0; j < kUnroll; j++)
                if (pb + 32 * j < p1)
                    sweep_one<WITH_BP, MULTI>(P, c.rd.qrow, d[j], sid[j], a0[j], a1[j], b0[j], b1[j], s_cnt, s_bp, cta_row);
        } else {
            // the step crosses a range boundary: one position at a time
            for (uint64_t pj = pb; pj < p1 && pj <= pb + 32 * (kUnroll - 1); pj += 32) {
                cursor_seek(P, c, pj, rcap);
                const uint64_t di = c.base + (pj - c.rlo);
                const uint2 d = __ldg(P.pos + di);
                uint2 a0, a1, b0, b1;
                bin_pair(P, c.tab, d.x, a0, a1);
                bin_pair(P, c.tab, d.y, b0, b1);
                sweep_one<WITH_BP, MULTI>(P, c.rd.qrow, d, __ldg(P.sid + di), a0, a1, b0, b1, s_cnt, s_bp, cta_row);
            }
        }
    }
}

template <bool WITH_BP, bool MULTI>
__global__ void __launch_bounds__(256, 5) k_sweep(SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long* s_bp = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + (WITH_BP ? (size_t)P.D * 8 : 0));
    const uint32_t lane = threadIdx.x & 31u;

    const uint32_t rcap = *P.rcount;
    const uint64_t total = P.rpos[rcap];
    if (P.smem_tally) {
        for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
            s_cnt[k] = 0;
            if (WITH_BP) s_bp[k] = 0;
        }
    }
    __syncthreads();
    if constexpr (MULTI) {
        // several rows: blocks pull block items (kCtaItems warp items each); the block's histogram
        // serves the row of the current item and is added to the outputs on a row change
        const uint64_t items = (total + P.chunk - 1) / P.chunk;
        multi_row_loop<true>(
            P, items, rcap,
            [&](uint32_t item, uint32_t row) {
                sweep_item<WITH_BP, true>(P, item, lane, rcap, total, s_cnt, s_bp, row);
            },
            [&](uint32_t row) { flush_row<WITH_BP>(P, row, s_cnt, s_bp); });
    } else {
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
            if ((uint64_t)item * P.chunk >= total) break;
            sweep_item<WITH_BP, false>(P, item, lane, rcap, total, s_cnt, s_bp, 0u);
        }
        if (P.smem_tally) {
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
                if (s_cnt[k]) atomicAdd(&P.counts[k], s_cnt[k]);
                if (WITH_BP && s_bp[k]) atomicAdd(&P.bp[k], s_bp[k]);
            }
        }
    }
}

// A pair candidate d of the run with query interval [qs, qe) and Q_SID qrow: when d.end > qs it
// adds 1 and min(ends) - max(starts) to cell (qrow, sid) — in the block's shared histograms (SMEM,
// one query row) or in the output matrix.
template <bool WITH_BP, bool SMEM, int MULTI>
__device__ __forceinline__ void pair_tally(const SweepParams& P, uint32_t qs, uint32_t qe, uint32_t qrow, uint2 d,
                                           uint32_t sid, uint32_t* s_cnt, unsigned long long* s_bp,
                                           uint32_t cta_row) {
    if (d.y <= qs) return;
    if (SMEM && (!MULTI || qrow == cta_row)) {
        atomicAdd(&s_cnt[sid], 1u);
        if (WITH_BP) add_u64_lo(&s_bp[sid], min(qe, d.y) - max(qs, d.x));
    } else {
        const uint64_t cell = (uint64_t)qrow * P.D + sid;
        atomicAdd(&P.counts[cell], 1u);
        if (WITH_BP) atomicAdd(&P.bp[cell], (unsigned long long)(min(qe, d.y) - max(qs, d.x)));
    }
}

// One step of the pair sweep position by position, each position's run found on its own by a
// galloping search from t.  Kept out of line: it runs only when a step holds 32 or more run
// boundaries (a stretch of empty runs), and inlined its registers would count against the whole
// kernel.
template <bool WITH_BP, bool SMEM, int MULTI>
__device__ __noinline__ void pairs_step_slow(const uint64_t* __restrict__ ppos, const PairSeg* __restrict__ psegs,
                                             const uint2* __restrict__ pos, const uint32_t* __restrict__ sidv,
                                             uint32_t* counts, unsigned long long* bp, uint32_t D, uint32_t t,
                                             uint32_t rcap, uint64_t pb, uint32_t span, uint32_t lane,
                                             uint32_t* s_cnt, unsigned long long* s_bp, uint32_t cta_row) {
    for (uint32_t o = lane; o <= span; o += 32) {
        const uint64_t pj = pb + o;
        const uint32_t tt = range_advance(ppos, t, rcap, pj);
        const PairSeg q = psegs[tt];
        const uint64_t di = q.base + (pj - __ldg(ppos + tt));
        const uint2 d = __ldg(pos + di);
        const uint32_t sid = __ldg(sidv + di);
        if (d.y <= q.qs) continue;
        if (SMEM && (!MULTI || q.qrow == cta_row)) {
            atomicAdd(&s_cnt[sid], 1u);
            if (WITH_BP) add_u64_lo(&s_bp[sid], min(q.qe, d.y) - max(q.qs, d.x));
        } else {
            const uint64_t cell = (uint64_t)q.qrow * D + sid;
            atomicAdd(&counts[cell], 1u);
            if (WITH_BP) atomicAdd(&bp[cell], (unsigned long long)(min(q.qe, d.y) - max(q.qs, d.x)));
        }
    }
}

// The pair sweep: the reference's scan (src/sweep/query.rs:104-115) over the candidate runs of the
// queries of pair ranges, every candidate read once by one lane (consecutive positions of a run are
// consecutive DB elements, so the loads coalesce).  A candidate d of query q overlaps when
// d.end > q.start (d.start < q.end and the look-back bound hold by construction of the run); it
// adds 1 and min(ends) - max(starts).
//
// A warp takes work items of `chunk` positions from the queue and walks each in steps of the
// 32 * kPairUnroll consecutive positions [pb, pend], lane l taking pb + l + 32 j.  The warp keeps
// the run t of the step's first position (uniform), so the choice between the forms below never
// splits the warp.  When the step lies in run t, every lane requests all its DB intervals and sids
// before using any.  When it spans several runs (about a quarter of the steps at hundreds of
// candidates per run), lane l holds the boundary ppos[t + 1 + l] of the following runs: a
// position's run is t plus the number of boundaries at or below it, counted over the few
// boundaries inside the step, and the run descriptors come from L1.
// One work item of the pair sweep (positions [item * chunk, (item + 1) * chunk) of the concatenated
// candidate runs), walked by one warp.
template <bool WITH_BP, bool SMEM, int MULTI>
__device__ __forceinline__ void pairs_item(const SweepParams& P, uint32_t item, uint32_t lane, uint32_t rcap,
                                           uint64_t total, uint32_t* s_cnt, unsigned long long* s_bp,
                                           uint32_t cta_row) {
    const uint64_t p0 = (uint64_t)item * P.chunk;
    const uint64_t p1 = min(p0 + P.chunk, total);
    uint32_t t;
    if (item < P.item_cap) {
        t = __ldg(P.item_t0 + item);
    } else {
        uint64_t lo = 0, hi = rcap;
        while (lo < hi) { uint64_t m = (lo + hi + 1) >> 1; if (__ldg(P.ppos + m) <= p0) lo = m; else hi = m - 1; }
        t = (uint32_t)lo;
    }
    uint64_t rlo = __ldg(P.ppos + t), rhi = __ldg(P.ppos + t + 1);
    PairSeg ps = P.psegs[t];
    for (uint64_t pb = p0; pb < p1; pb += 32 * kPairUnroll) {
        const uint64_t pend = min(pb + 32 * kPairUnroll, p1) - 1;
        const uint32_t span = (uint32_t)(pend - pb);
        if (pb >= rhi) {
            t = range_advance(P.ppos, t, rcap, pb);
            rlo = __ldg(P.ppos + t);
            rhi = __ldg(P.ppos + t + 1);
            ps = P.psegs[t];
        }
        const uint64_t base0 = ps.base - rlo + pb;  // element of offset 0 when it lies in run t
        if (pend < rhi) {
            uint2 d[kPairUnroll];
            uint32_t sid[kPairUnroll];
#pragma unroll
            for (uint32_t j = 0; j < kPairUnroll; j++) {
                const uint32_t o = lane + 32 * j;
                if (o <= span) {
                    d[j] = __ldg(P.pos + base0 + o);
                    sid[j] = __ldg(P.sid + base0 + o);
                } else {
                    d[j] = make_uint2(0, 0);  // never a hit: d.y = 0 <= qs
                    sid[j] = 0;
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < kPairUnroll; j++)
                pair_tally<WITH_BP, SMEM, MULTI>(P, ps.qs, ps.qe, ps.qrow, d[j], sid[j], s_cnt, s_bp, cta_row);
            continue;
        }
        // lane l: boundary ppos[t + 1 + l] as an offset from pb (> 0, since run t holds pb);
        // offsets inside the step fit 32 bits
        const uint64_t B = (uint64_t)t + 1 + lane <= rcap ? __ldg(P.ppos + t + 1 + lane) : ~0ull;
        const uint32_t rel = B - pb < 0xffffffffull ? (uint32_t)(B - pb) : 0xffffffffu;
        const uint32_t nb = __popc(__ballot_sync(0xffffffffu, rel <= span));
        if (nb == 32) {
            pairs_step_slow<WITH_BP, SMEM, MULTI>(P.ppos, P.psegs, P.pos, P.sid, P.counts, P.bp, P.D, t, rcap, pb, span,
                                           lane, s_cnt, s_bp, cta_row);
            continue;  // the next step starts past rhi: range_advance finds its run
        }
        uint32_t k[kPairUnroll];  // position lane + 32 j lies in run t + k[j]
#pragma unroll
        for (uint32_t j = 0; j < kPairUnroll; j++) k[j] = 0;
        for (uint32_t i = 0; i < nb; i++) {  // rel[0..nb) are the boundaries inside the step
            const uint32_t bv = __shfl_sync(0xffffffffu, rel, i);
#pragma unroll
            for (uint32_t j = 0; j < kPairUnroll; j++) k[j] += bv <= lane + 32 * j ? 1u : 0u;
        }
        uint2 d[kPairUnroll];
        uint32_t sid[kPairUnroll];
#pragma unroll
        for (uint32_t j = 0; j < kPairUnroll; j++) {
            // run t + k (k > 0) starts at offset rel[k - 1]; t + k < rcap since ppos[rcap] = total > pend
            const uint32_t o = lane + 32 * j;
            const uint32_t rb = __shfl_sync(0xffffffffu, rel, k[j] ? k[j] - 1 : 0);
            if (o <= span) {
                const uint64_t di = k[j] ? __ldg(&P.psegs[t + k[j]].base) + (o - rb) : base0 + o;
                d[j] = __ldg(P.pos + di);
                sid[j] = __ldg(P.sid + di);
            } else {
                d[j] = make_uint2(0, 0);
                sid[j] = 0;
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < kPairUnroll; j++) {
            const PairSeg* q = P.psegs + t + k[j];
            pair_tally<WITH_BP, SMEM, MULTI>(P, __ldg(&q->qs), __ldg(&q->qe),
                                             (SMEM && !MULTI) ? 0u : __ldg(&q->qrow), d[j], sid[j], s_cnt, s_bp,
                                             cta_row);
        }
        // the run of the next step's first position pend + 1, from the boundaries in hand (at
        // least one boundary, ppos[t + 1] <= pend, lies at or below it)
        const uint32_t kn = __popc(__ballot_sync(0xffffffffu, rel <= span + 1));
        if (pend + 1 < p1 && kn < 32) {
            t += kn;
            rlo = __ldg(P.ppos + t);
            rhi = __ldg(P.ppos + t + 1);
            ps = P.psegs[t];
        }
    }
}

template <bool WITH_BP, bool SMEM, int MULTI>
__global__ void __launch_bounds__(256, MULTI ? 6 : 8) k_pairs(SweepParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long* s_bp = reinterpret_cast<unsigned long long*>(smem);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + (WITH_BP ? (size_t)P.D * 8 : 0));
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t rcap = *P.pcount;
    const uint64_t total = P.ppos[rcap];
    if (SMEM)
        for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
            s_cnt[k] = 0;
            if (WITH_BP) s_bp[k] = 0;
        }
    __syncthreads();
    if constexpr (MULTI) {
        // several rows: block items, the histogram serves one row at a time (as k_sweep)
        const uint64_t items = (total + P.chunk - 1) / P.chunk;
        multi_row_loop<false>(
            P, items, rcap,
            [&](uint32_t item, uint32_t row) {
                pairs_item<WITH_BP, true, 1>(P, item, lane, rcap, total, s_cnt, s_bp, row);
            },
            [&](uint32_t row) { flush_row<WITH_BP>(P, row, s_cnt, s_bp); });
    } else {
        for (;;) {
            uint32_t item = 0;
            if (lane == 0) item = atomicAdd(P.queue, 1u);
            item = __shfl_sync(0xffffffffu, item, 0);
            if ((uint64_t)item * P.chunk >= total) break;
            pairs_item<WITH_BP, SMEM, 0>(P, item, lane, rcap, total, s_cnt, s_bp, 0u);
        }
        if (SMEM) {
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < P.D; k += blockDim.x) {
                if (s_cnt[k]) atomicAdd(&P.counts[k], s_cnt[k]);
                if (WITH_BP && s_bp[k]) atomicAdd(&P.bp[k], s_bp[k]);
            }
        }
    }
}

// `--intervals` mode (query_sweep_pairs, src/sweep/query.rs:11-41): every overlapping pair of the
// candidate runs, listed in the order of the pair work space (layer slot, shard, row, query start,
// DB start).  Item i = positions [i * chunk, (i + 1) * chunk) is walked by one warp, 32 positions
// per step: the count pass stores the item's hits, the emit pass writes them from the item's
// offset (an exclusive scan of the counts) at their ballot ranks, so the list needs no atomics and
// comes out in the same order every time.
template <bool EMIT>
__global__ void __launch_bounds__(256) k_pair_list(const uint64_t* __restrict__ ppos,
                                                   const uint32_t* __restrict__ pcount,
                                                   const PairSeg* __restrict__ psegs, const uint2* __restrict__ pos,
                                                   const uint32_t* __restrict__ sid, uint64_t items, uint32_t chunk,
                                                   uint64_t* __restrict__ item_hits,
                                                   const uint64_t* __restrict__ item_base, rgl_pair* __restrict__ out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t rcap = *pcount;
    const uint64_t total = ppos[rcap];
    for (uint64_t item = warp; item < items; item += nwarps) {
        const uint64_t p0 = item * chunk, p1 = min(p0 + chunk, total);
        uint64_t lo = 0, hi = rcap;  // last run t with ppos[t] <= p0
        while (lo < hi) {
            const uint64_t m = (lo + hi + 1) >> 1;
            if (__ldg(ppos + m) <= p0) lo = m; else hi = m - 1;
        }
        uint32_t t = (uint32_t)lo;
        uint64_t rhi = __ldg(ppos + t + 1), rlo = __ldg(ppos + t);
        PairSeg ps = psegs[t];
        const uint64_t base = EMIT ? item_base[item] : 0;
        uint64_t done = 0;
        for (uint64_t s = p0; s < p1; s += 32) {
            const uint64_t p = s + lane;
            bool hit = false;
            uint2 d = make_uint2(0, 0);
            uint64_t di = 0;
            if (p < p1) {
                if (p >= rhi) {
                    t = range_advance(ppos, t, rcap, p);
                    rlo = __ldg(ppos + t);
                    rhi = __ldg(ppos + t + 1);
                    ps = psegs[t];
                }
                di = ps.base + (p - rlo);
                d = __ldg(pos + di);
                hit = d.y > ps.qs;
            }
            const uint32_t ballot = __ballot_sync(0xffffffffu, hit);
            if (EMIT && hit) {
                const uint32_t rank = __popc(ballot & ((1u << lane) - 1u));
                rgl_pair r;
                r.query_start = ps.qs;
                r.query_end = ps.qe;
                r.db_start = d.x;
                r.db_end = d.y;
                r.row = ps.qrow;
                r.sid = __ldg(sid + di);
                r.shard = ps.shard;
                r.intersection_bp = min(ps.qe, d.y) - max(ps.qs, d.x);
                out[base + done + rank] = r;
            }
            done += __popc(ballot);
        }
        if (!EMIT && lane == 0) item_hits[item] = done;
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
    // second stream for the independent chains of a run (the end-key sort, the prefix sums of the
    // starts and ends, the rank tables), forked from and joined back into `stream`
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int num_sms = 148;
    DevBuf iv, blk_off, blk_shard, key_a, key_b, val_a, val_b, ekey_a, ekey_b;
    DevBuf starts, ends, seg, segflag, segnum, seg_begin, ps_in, pe_in, ps, pe;
    DevBuf lo, hi, maxhi, rflag, ridx, ranges, rlen, rpos, cub_tmp, small, out_counts, out_bp, item_r0;
    DevBuf segtab, tab_len, tab_off, tab_s, tab_e, tab_xs, tab_xe, tab2;
    DevBuf cl, pc, method, plen, ppos, psegs, item_t0, seg_need, tl, scan_sums;
    DevBuf cub_tmp2, scan_sums2;  // the side stream's own scratch
    DevBuf sortplan;  // block-local sort: order flags, tile and merge-chunk prefix counts, two pass words
    DevBuf sort_tab, sort_rank;  // its segment-order layout, for the single-call entry points
    DevBuf item_hits, item_base, pairs;  // intervals mode
    DevBuf bt_off, bt_shard, acc;  // batched form: sub-batch block tables (offsets; shards then rows), stats
    uint32_t* h_small = nullptr;  // pinned mirror of `small`
    unsigned long long* h_acc = nullptr;  // pinned mirror of `acc`
    uint64_t ws_sig = 0;          // changes whenever a workspace buffer is reallocated
    // the CUDA graph of the last batch run with RGL_BF_GRAPH, replayed while the batch is unchanged
    struct GraphCache {
        std::vector<uint64_t> key;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        DevBuf t_off, t_shard;  // the graph's own copies of the block tables
        uint32_t nodes = 0, launches = 0, subs = 0;
    } gc;
    // host-input batches: two staging buffers filled on a copy stream while the other is swept
    DevBuf stage[2];
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_used[2] = {nullptr, nullptr};
    bool has_tuned = false;       // rgl_batch_autotune result
    rgl_query_opts tuned{};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t res_n = 0;           // the workspace covers runs of res_n intervals, res_rows rows and
    uint32_t res_rows = 0;        // res_blk blocks (every buffer's size depends on one of the three)
    uint32_t res_blk = 0;
    bool ws_ready = false;        // res_* describe the workspace (set by the first full sizing)
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

// Default work-item size of runs with several output rows.
constexpr uint32_t kMultiRowChunk = 8192;

// Runs up to this many query intervals chain their kernels with programmatic dependent launch.
constexpr uint64_t kPdlMaxIntervals = 1ull << 21;

// Query intervals per pipeline run: the rank tables (up to 10 entries per interval) use 31-bit offsets.
constexpr uint64_t kMaxRunIntervals = 200000000ull;

// Sizes every workspace buffer for a run of n query intervals, `rows` output rows and nblk input
// blocks.  With plan != nullptr nothing is allocated: *plan receives the bytes that growing the
// buffers would add (a buffer grows by freeing and reallocating it at the larger size).
int size_workspace(rgl_context* c, uint64_t n, uint32_t rows, uint32_t nblk, uint64_t* plan) {
    rgl_index* idx = c->idx;
    if (n > kMaxRunIntervals) return fail(RGL_ERR_INVALID_ARGUMENT, "at most 200,000,000 query intervals per run");
    const uint64_t ns = std::max<uint32_t>(idx->num_slots, 1);
    const uint64_t tot = n * ns;
    if (plan) *plan = 0;
    if (c->ws_ready && n <= c->res_n && rows <= c->res_rows && nblk <= c->res_blk) return RGL_OK;  // nothing grows
    struct Sizer {
        uint64_t* plan;
        int ensure_in(DevBuf& b, size_t bytes) {
            if (!plan) return b.ensure(bytes);
            if (bytes > b.cap) *plan += bytes - b.cap;
            return RGL_OK;
        }
    } z{plan};
    RGL_TRY(z.ensure_in(c->iv, n * sizeof(rgl_interval) + 16));
    RGL_TRY(z.ensure_in(c->blk_off, (nblk + 1) * 8ull));
    RGL_TRY(z.ensure_in(c->blk_shard, (nblk + 1) * 4ull));
    RGL_TRY(z.ensure_in(c->sortplan, (4ull * nblk + 8) * 4));
    // the block tables of a run with rows taken from the blocks (offsets, the sort's segment-order
    // offsets and destinations; shards, rows, ranks), sized here so that no run reallocates them
    RGL_TRY(z.ensure_in(c->bt_off, 3ull * (nblk + 1) * 8 + 8));
    RGL_TRY(z.ensure_in(c->bt_shard, 3ull * (nblk + 1) * 4 + 4));
    RGL_TRY(z.ensure_in(c->key_a, n * 8 + 8));
    RGL_TRY(z.ensure_in(c->key_b, n * 8 + 8));
    RGL_TRY(z.ensure_in(c->val_a, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->val_b, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->ekey_a, n * 8 + 8));
    RGL_TRY(z.ensure_in(c->ekey_b, n * 8 + 8));
    RGL_TRY(z.ensure_in(c->starts, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->ends, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->seg, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->segflag, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->segnum, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->seg_begin, n * 4 + 4));
    RGL_TRY(z.ensure_in(c->seg_need, n * 8 + 8));
    RGL_TRY(z.ensure_in(c->ps_in, n * 8 + 16));
    RGL_TRY(z.ensure_in(c->pe_in, n * 8 + 16));
    RGL_TRY(z.ensure_in(c->ps, n * 8 + 16));
    RGL_TRY(z.ensure_in(c->pe, n * 8 + 16));
    RGL_TRY(z.ensure_in(c->lo, tot * 4 + 4));
    RGL_TRY(z.ensure_in(c->hi, tot * 4 + 4));
    RGL_TRY(z.ensure_in(c->maxhi, tot * 4 + 4));
    RGL_TRY(z.ensure_in(c->rflag, tot * 4 + 8));
    RGL_TRY(z.ensure_in(c->ridx, tot * 4 + 8));
    RGL_TRY(z.ensure_in(c->ranges, tot * sizeof(RangeDesc) + sizeof(RangeDesc)));
    RGL_TRY(z.ensure_in(c->rlen, tot * 8 + 16));
    RGL_TRY(z.ensure_in(c->rpos, tot * 8 + 16));
    RGL_TRY(z.ensure_in(c->small, 256));
    RGL_TRY(z.ensure_in(c->item_r0, kItemCap * 4));
    RGL_TRY(z.ensure_in(c->item_t0, kItemCap * 4));
    RGL_TRY(z.ensure_in(c->cl, tot * 8 + 16));
    RGL_TRY(z.ensure_in(c->pc, tot * 8 + 16));
    RGL_TRY(z.ensure_in(c->method, tot + 16));
    RGL_TRY(z.ensure_in(c->tl, tot * 4 + 8));
    RGL_TRY(z.ensure_in(c->scan_sums, (std::max<uint64_t>(tot, 10 * n + 16) / kScanTile + 4) * 8));
    RGL_TRY(z.ensure_in(c->scan_sums2, (10 * n + 16) / kScanTile * 8 + 32));
    RGL_TRY(z.ensure_in(c->plen, tot * 8 + 16));
    RGL_TRY(z.ensure_in(c->ppos, tot * 8 + 16));
    RGL_TRY(z.ensure_in(c->psegs, tot * sizeof(PairSeg) + sizeof(PairSeg)));
    RGL_TRY(z.ensure_in(c->segtab, (n + 1) * sizeof(SegTab)));
    RGL_TRY(z.ensure_in(c->tab_len, (n + 2) * 4));
    RGL_TRY(z.ensure_in(c->tab_off, (n + 2) * 4));
    RGL_TRY(z.ensure_in(c->tab_s, (10 * n + 18) * 4));
    RGL_TRY(z.ensure_in(c->tab_e, (10 * n + 18) * 4));
    RGL_TRY(z.ensure_in(c->tab2, (10 * n + 18) * 8));
    RGL_TRY(z.ensure_in(c->tab_xs, (10 * n + 16) * 4));
    RGL_TRY(z.ensure_in(c->tab_xe, (10 * n + 16) * 4));
    RGL_TRY(z.ensure_in(c->acc, 64));
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
    cub::DeviceScan::InclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)(10 * n + 16), c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nn + 1, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    cub::DeviceSelect::Flagged(nullptr, b, thrust::counting_iterator<uint32_t>(0), (const uint32_t*)nullptr,
                               (uint32_t*)nullptr, (uint32_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, nn + 1, c->stream);
    need = std::max(need, b);
    cub::DeviceReduce::Sum(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, nt, c->stream);
    need = std::max(need, b);
    RGL_TRY(z.ensure_in(c->cub_tmp, need + 256));
    RGL_TRY(z.ensure_in(c->cub_tmp2, need + 256));
    if (rows) {
        RGL_TRY(z.ensure_in(c->out_counts, (uint64_t)rows * idx->num_sources * 4 + 16));
        RGL_TRY(z.ensure_in(c->out_bp, (uint64_t)rows * idx->num_sources * 8 + 16));
    }
    if (plan) return RGL_OK;
    c->res_n = std::max(c->res_n, n);
    c->res_rows = std::max(c->res_rows, rows);
    c->res_blk = std::max(c->res_blk, nblk);
    c->ws_ready = true;
    uint64_t sig = 1469598103934665603ull;
    for (DevBuf* b : {&c->iv, &c->key_a, &c->key_b, &c->val_a, &c->val_b, &c->ekey_a, &c->ekey_b, &c->starts,
                      &c->ends, &c->seg, &c->segflag, &c->segnum, &c->seg_begin, &c->ps_in, &c->pe_in, &c->ps,
                      &c->pe, &c->lo, &c->hi, &c->maxhi, &c->rflag, &c->ridx, &c->ranges, &c->rlen, &c->rpos,
                      &c->cub_tmp, &c->small, &c->item_r0, &c->item_t0, &c->segtab, &c->tab_len, &c->tab_off,
                      &c->tab_s, &c->tab_e, &c->tab_xs, &c->tab_xe, &c->tab2, &c->cl, &c->pc, &c->method, &c->tl, &c->scan_sums, &c->plen, &c->ppos, &c->psegs,
                      &c->seg_need, &c->acc, &c->cub_tmp2, &c->scan_sums2, &c->sortplan})
        sig = (sig ^ (uint64_t)(uintptr_t)b->p ^ ((uint64_t)b->cap << 17)) * 1099511628211ull;
    c->ws_sig = sig;
    return RGL_OK;
}

int ensure_workspace(rgl_context* c, uint64_t n, uint32_t rows, uint32_t nblk) {
    return size_workspace(c, n, rows, nblk, nullptr);
}

inline unsigned grid_for(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

struct Launch {
    uint32_t chunk, ctas_per_sm, block, pair_ratio;
};

Launch pick_launch(const rgl_query_opts* o) {
    Launch l{1024, 8, 256, 4};
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
        // the pipeline's device counters (small[4..5] union, [9] ranges, [10..11] / [12..13] rank /
        // pair work) were copied to h_small after the run
        stats->ranges = c->last_n ? c->h_small[9] : 0;
        uint64_t T = 0;
        if (c->last_n) std::memcpy(&T, c->h_small + 4, 8);
        stats->db_swept = T;
        uint64_t TR = 0, TP = 0;
        if (c->last_n) {
            std::memcpy(&TR, c->h_small + 10, 8);
            std::memcpy(&TP, c->h_small + 12, 8);
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

// Exclusive scan of in[0, *n_ptr) into out (with out[n] = total), n <= cap; returns the launches.
// Launches a short kernel of a pipeline chain: with `pdl` its PDL variant (which begins with
// pdl_wait()) with programmatic stream serialization, so that it may be scheduled while the previous
// grid of the stream is finishing; else its plain variant.  PDL is used for small runs, where the
// launch latency between the short kernels of a chain is a visible share of the run.
template <typename... K, typename... A>
cudaError_t launch_chain(bool pdl, void (*with_pdl)(K...), void (*plain)(K...), dim3 grid, dim3 block, size_t smem,
                         cudaStream_t st, A&&... args) {
    if (!pdl) {
        plain<<<grid, block, smem, st>>>(std::forward<A>(args)...);  // errors surface at the next check
        return cudaSuccess;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, with_pdl, std::forward<A>(args)...);
}

// `sums` holds cap / kScanTile + 1 tile sums (one buffer per stream that scans concurrently).
template <typename Tin, typename Tout>
uint32_t scan_dev(Tout* sums, const Tin* in, Tout* out, const uint32_t* n_ptr, uint64_t cap, cudaStream_t st,
                  bool pdl) {
    const unsigned grid = (unsigned)std::min<uint64_t>(cap / kScanTile + 1, 148ull * 8);
    (void)launch_chain(pdl, k_scan_reduce<Tin, Tout, true>, k_scan_reduce<Tin, Tout, false>, grid, kScanThreads, 0,
                     st, in, n_ptr, sums);
    (void)launch_chain(pdl, k_scan_tops<Tout, true>, k_scan_tops<Tout, false>, 1, 1024, 0, st, sums, n_ptr, out);
    (void)launch_chain(pdl, k_scan_apply<Tin, Tout, true>, k_scan_apply<Tin, Tout, false>, grid, kScanThreads, 0, st,
                     in, out, n_ptr, sums);
    return 3;
}

// `to` waits for everything enqueued on `from` so far.
int stream_after(cudaStream_t to, cudaStream_t from, cudaEvent_t e) {
    RGL_CUDA(cudaEventRecord(e, from));
    RGL_CUDA(cudaStreamWaitEvent(to, e, 0));
    return RGL_OK;
}

// Shape of a run's block-local key sort, from the host's block offsets.
struct LocalSort {
    uint64_t max_block = 0;  // the largest block: sets the number of merge passes
    uint64_t tiles = 0;      // tiles of kBlockSortCap intervals over all blocks
    uint64_t chunks = 0;     // merge chunks of the blocks of more than one tile
    // When the blocks are not in segment order (file-major blocks of several rows), the sorted keys
    // are laid out segment by segment, as a device-wide sort would lay them out, so that the sweeps
    // take every row's work on one chromosome together: block b's keys go to [dst[b], dst[b] +
    // cnt_b), its rank in segment order is idx[b], and soff (nblk + 1) are the offsets of the blocks
    // in that order.  Empty: the blocks are in segment order already.
    std::vector<uint64_t> soff, dst;
    std::vector<uint32_t> idx;
};

// Input of one pipeline run: n intervals at `iv` (device), block b = [blk_off[b], blk_off[b+1]) on
// shard blk_shard[b] (both tables on the device), rows [row_base, row_base + rows) of the output.
struct PipeIn {
    const rgl_interval* iv;
    uint64_t n;
    uint32_t rows, row_base, nblk;
    const uint64_t* blk_off;
    const uint32_t* blk_shard;
    const uint32_t* blk_row;  // optional: the row every interval of the block must carry
    int row_from_block = 0;   // 1: rows come from blk_row, interval sids are ignored
    int block_local = 0;      // 1: one segment per block, no segment in two blocks (block-local key sort)
    LocalSort ls;             // with block_local: the sort's tile and merge-chunk counts
    // with block_local and a segment-order layout: device copies of ls.soff, ls.dst, ls.idx
    const uint64_t* sort_off = nullptr;
    const uint64_t* sort_dst = nullptr;
    const uint32_t* sort_idx = nullptr;
    uint32_t region_bits = 0; // > 0: segments are (shard, 2^region_bits-bp region of the start, row)
};

// Whether a run's blocks allow the block-local key sort: with one row, or rows taken from the
// blocks, every block is one segment, and they must be distinct.  off: nblk + 1 host offsets; row:
// the blocks' rows (null: row 0 of one row).  *ls receives the shape of the sort.
bool blocks_local(uint32_t nblk, const uint64_t* off, const uint32_t* shard, const uint32_t* row, uint32_t rows,
                  uint32_t row_base, LocalSort* ls) {
    *ls = LocalSort();
    if (!row && rows != 1) return false;
    std::vector<std::pair<uint64_t, uint32_t>> segs;  // (segment, block) of the non-empty blocks
    segs.reserve(nblk);
    LocalSort t;
    bool ordered = true;
    for (uint32_t b = 0; b < nblk; b++) {
        const uint64_t cnt = off[b + 1] - off[b];
        t.max_block = std::max(t.max_block, cnt);
        t.tiles += sort_tiles(cnt);
        t.chunks += merge_chunks(cnt);
        const uint64_t sg = (uint64_t)shard[b] * rows + (row ? row[b] - row_base : 0u);
        if (cnt) {
            if (!segs.empty() && sg < segs.back().first) ordered = false;
            segs.push_back({sg, b});
        }
    }
    std::vector<std::pair<uint64_t, uint32_t>> sorted(segs);
    std::stable_sort(sorted.begin(), sorted.end(),
                     [](const std::pair<uint64_t, uint32_t>& a, const std::pair<uint64_t, uint32_t>& b) {
                         return a.first < b.first;
                     });
    for (size_t k = 1; k < sorted.size(); k++)
        if (sorted[k].first == sorted[k - 1].first) return false;  // a segment in two blocks
    if (!ordered) {
        // empty blocks keep their place in the order (rank) and take no room
        std::vector<uint32_t> order;
        order.reserve(nblk);
        size_t k = 0;
        for (uint32_t b = 0; b < nblk; b++)
            if (off[b + 1] == off[b]) order.push_back(b);
        std::vector<uint32_t> empties(order);
        order.clear();
        for (const auto& e : sorted) order.push_back(e.second);
        order.insert(order.end(), empties.begin(), empties.end());
        t.soff.assign(nblk + 1, 0);
        t.dst.assign(nblk + 1, 0);
        t.idx.assign(nblk + 1, 0);
        uint64_t at = 0;
        for (k = 0; k < order.size(); k++) {
            const uint32_t b = order[k];
            t.soff[k] = at;
            t.dst[b] = at;
            t.idx[b] = (uint32_t)k;
            at += off[b + 1] - off[b];
        }
        t.soff[nblk] = at;
        t.dst[nblk] = at;
    }
    *ls = std::move(t);
    return true;
}

// What a run does besides the sweep: the single-call entry points zero their rows, reset the error
// word and record stats events; the sub-batches of a batched call leave all of that to the caller
// and add their stats into a device accumulator.
struct PipeMode {
    bool zero_out = true;
    bool reset_err = true;
    bool events = true;  // stats events and sweep timing (off inside a graph capture)
    bool no_sweep = false;  // stop once the pair work space (ppos, psegs) is laid out
    unsigned long long* acc = nullptr;
};

__global__ void k_acc_stats(unsigned long long* acc, const uint32_t* ranges, const unsigned long long* uni,
                            const unsigned long long* rank_pos, const unsigned long long* pair_cand, uint32_t n) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        acc[0] += *ranges;
        acc[1] += *uni;
        acc[2] += *rank_pos;
        acc[3] += *pair_cand;
        acc[4] += n;
    }
}

// Runs steps 1-5 of the pipeline on the context stream, with no host synchronisation.
int run_pipeline(rgl_context* c, const PipeIn& in, const rgl_query_opts* opts, uint32_t* d_counts,
                 unsigned long long* d_bp, rgl_query_stats* stats, const PipeMode& mode = PipeMode()) {
    rgl_index* idx = c->idx;
    cudaStream_t st = c->stream;
    const uint32_t D = idx->num_sources;
    const uint32_t ns = idx->num_slots;
    const uint32_t n = (uint32_t)in.n;
    const uint32_t rows = in.rows;
    Launch L = pick_launch(opts);
    // several rows: the block items flush their row histogram, so larger work items pay (measured
    // on the 2e9-interval database: 1024 -> 8192 positions, sweeps 3.45 -> 2.46 s per 4,096 files)
    if (rows > 1 && !(opts && opts->chunk)) L.chunk = kMultiRowChunk;
    const bool with_bp = d_bp != nullptr && !(opts && (opts->flags & RGL_QF_NO_OVERLAP));
    const bool ev = mode.events && stats;
    const bool pdl = in.n <= kPdlMaxIntervals;

    uint32_t* d_small = c->small.as<uint32_t>();  // [0] error bits, [1] queue, [2..] scratch
    if (mode.reset_err) RGL_CUDA(cudaMemsetAsync(d_small, 0, 64, st));
    else RGL_CUDA(cudaMemsetAsync(d_small + 1, 0, 60, st));
    if (mode.zero_out) {
        if (d_counts) RGL_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)rows * D * 4, st));
        if (d_bp) RGL_CUDA(cudaMemsetAsync(d_bp, 0, (size_t)rows * D * 8, st));
    }
    if (n == 0 || ns == 0) {
        c->last_n = 0;
        c->last_tot = 0;
        c->last_launches = 0;
        if (stats) std::memset(stats, 0, sizeof(*stats));
        if (mode.reset_err) RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
        return RGL_OK;
    }
    // key width: segment = shard * rows + row
    const uint32_t rb = in.region_bits;
    if (rb && (rb < 16 || rb > 31)) return fail(RGL_ERR_INVALID_ARGUMENT, "region bits must be in [16, 31]");
    const uint64_t nreg = rb ? (1ull << (32 - rb)) : 1ull;
    uint64_t nseg = (uint64_t)idx->num_shards * nreg * rows;
    int segbits = 1;
    while (segbits < 32 && (1ull << segbits) < nseg) segbits++;
    if (nseg >= (1ull << 32))
        return fail(RGL_ERR_INVALID_ARGUMENT, "num_shards x regions x num_rows must be < 2^32");
    const uint32_t sps = (uint32_t)(nreg * rows);  // segments per shard

    if (ev) RGL_CUDA(cudaEventRecord(c->ev[0], st));
    // Two streams: `st` carries the chain from the sorted starts to the sweeps, `sd` the chains that
    // only the rank sweep needs (the end-key sort and unpack, the prefix sums of starts and ends,
    // the rank tables), so that the small kernels of both overlap; `sd` is joined back before the
    // sweeps.
    cudaStream_t sd = c->side;
    uint32_t launches = 0;
    // block-local sort with a segment-order layout: callers that did not upload its tables (the
    // single-call entry points, never inside a graph capture) have them uploaded here
    const uint64_t* sort_off = in.sort_off;
    const uint64_t* sort_dst = in.sort_dst;
    const uint32_t* sort_idx = in.sort_idx;
    if (in.block_local && !in.ls.dst.empty() && !sort_dst) {
        const uint64_t nb1 = (uint64_t)in.nblk + 1;
        RGL_TRY(c->sort_tab.ensure(2 * nb1 * 8));
        RGL_TRY(c->sort_rank.ensure(nb1 * 4));
        RGL_CUDA(cudaMemcpyAsync(c->sort_tab.p, in.ls.soff.data(), nb1 * 8, cudaMemcpyHostToDevice, st));
        RGL_CUDA(cudaMemcpyAsync(c->sort_tab.as<uint64_t>() + nb1, in.ls.dst.data(), nb1 * 8, cudaMemcpyHostToDevice,
                                 st));
        RGL_CUDA(cudaMemcpyAsync(c->sort_rank.p, in.ls.idx.data(), nb1 * 4, cudaMemcpyHostToDevice, st));
        sort_off = c->sort_tab.as<uint64_t>();
        sort_dst = sort_off + nb1;
        sort_idx = c->sort_rank.as<uint32_t>();
    }
    // block-local sort: per-block order flags ([0, nblk) starts, [nblk, 2 nblk) ends), then the
    // tile and merge-chunk prefix counts
    uint32_t* d_unsorted = c->sortplan.as<uint32_t>();
    uint32_t* d_tile_pre = d_unsorted + 2ull * in.nblk;
    uint32_t* d_chunk_pre = d_tile_pre + in.nblk + 1;
    if (in.block_local) RGL_CUDA(cudaMemsetAsync(d_unsorted, 0, 2ull * in.nblk * 4, st));
    k_expand_keys<<<grid_for(n, 256), 256, 0, st>>>(n, in.iv, in.blk_off, in.blk_shard, in.blk_row,
                                                    in.row_from_block, in.nblk, rows, in.row_base, rb,
                                                    c->key_a.as<uint64_t>(), c->val_a.as<uint32_t>(),
                                                    c->ekey_a.as<uint64_t>(), d_small,
                                                    in.block_local ? d_unsorted : nullptr,
                                                    in.block_local ? sort_dst : nullptr,
                                                    in.block_local ? sort_idx : nullptr);
    launches++;
    // the sort's view of the blocks: their offsets in the layout the keys were written in
    const uint64_t* soff = sort_dst ? sort_off : in.blk_off;
    const uint32_t passes = in.block_local ? sort_passes(in.ls.max_block) : 0u;
    if (in.block_local)  // the plan (before the fork), then the end keys here and the start keys there
        launches += block_sort_enqueue(in.nblk, soff, 0, 0, 0, d_tile_pre, d_chunk_pre, nullptr, nullptr, nullptr,
                                       nullptr, nullptr, nullptr, st, true);
    RGL_TRY(stream_after(sd, st, c->ev_fork));
    size_t tb = c->cub_tmp2.cap;
    if (in.block_local) {
        launches += block_sort_enqueue(in.nblk, soff, in.ls.tiles, in.ls.chunks, passes, d_tile_pre, d_chunk_pre,
                                       d_unsorted + in.nblk, c->ekey_a.as<uint64_t>(), nullptr,
                                       c->ekey_b.as<uint64_t>(), nullptr, d_chunk_pre + in.nblk + 2, sd, false);
        launches += block_sort_enqueue(in.nblk, soff, in.ls.tiles, in.ls.chunks, passes, d_tile_pre, d_chunk_pre,
                                       d_unsorted, c->key_a.as<uint64_t>(), c->val_a.as<uint32_t>(),
                                       c->key_b.as<uint64_t>(), c->val_b.as<uint32_t>(), d_chunk_pre + in.nblk + 1, st,
                                       false);
    } else {
        RGL_CUDA(cub::DeviceRadixSort::SortKeys(c->cub_tmp2.p, tb, c->ekey_a.as<uint64_t>(), c->ekey_b.as<uint64_t>(),
                                                (int)n, 0, 32 + segbits, sd));
        tb = c->cub_tmp.cap;
        RGL_CUDA(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tb, c->key_a.as<uint64_t>(), c->key_b.as<uint64_t>(),
                                                 c->val_a.as<uint32_t>(), c->val_b.as<uint32_t>(), (int)n, 0,
                                                 32 + segbits, st));
    }
    // the side stream goes on with the ends (their prefix sums), the main one with the starts
    k_unpack_ends<<<grid_for(n + 1, 256), 256, 0, sd>>>(n, c->ekey_b.as<uint64_t>(), c->ends.as<uint32_t>(),
                                                        c->pe_in.as<uint64_t>());
    tb = c->cub_tmp2.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp2.p, tb, c->pe_in.as<uint64_t>(), c->pe.as<uint64_t>(),
                                           (int)n + 1, sd));
    k_unpack_starts<<<grid_for(n + 1, 256), 256, 0, st>>>(n, c->key_b.as<uint64_t>(), c->starts.as<uint32_t>(),
                                                          c->seg.as<uint32_t>(), c->segflag.as<uint32_t>(),
                                                          c->ps_in.as<uint64_t>());
    launches += 2;
    RGL_TRY(stream_after(sd, st, c->ev_fork));
    tb = c->cub_tmp2.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp2.p, tb, c->ps_in.as<uint64_t>(), c->ps.as<uint64_t>(),
                                           (int)n + 1, sd));
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::InclusiveSum(c->cub_tmp.p, tb, c->segflag.as<uint32_t>(), c->segnum.as<uint32_t>(),
                                           (int)n, st));
    k_seg_begin<<<grid_for(n, 256), 256, 0, st>>>(n, c->segflag.as<uint32_t>(), c->segnum.as<uint32_t>(),
                                                  c->seg_begin.as<uint32_t>());
    launches++;
    RGL_CUDA(cudaMemsetAsync(c->seg_need.p, 0, (size_t)(n + 1) * 8, st));
    const uint64_t tot = (uint64_t)n * ns;
    if (tot + 1 >= (1ull << 31)) {
        RGL_TRY(stream_after(st, sd, c->ev_join));
        return fail(RGL_ERR_INVALID_ARGUMENT, "query intervals x layer slots must be < 2^31 per run");
    }
    k_lohi<<<dim3(grid_for(n, 256), ns), 256, 0, st>>>(n, ns, sps, c->starts.as<uint32_t>(), c->val_b.as<uint32_t>(),
                                                c->seg.as<uint32_t>(), idx->d_slot, idx->d_layers, idx->d_pos,
                                                idx->d_btab, c->lo.as<uint32_t>(), c->hi.as<uint32_t>(),
                                                c->rflag.as<uint32_t>());
    launches++;
    // live runs: compaction of the (K, query) entries with a non-empty candidate run (flags from
    // k_lohi) in one pass: tl[c] = t of the c-th live entry, *Lp = their number
    uint32_t* Lp = d_small + 8;  // live runs L
    uint32_t* Rp = d_small + 9;  // ranges R
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceSelect::Flagged(c->cub_tmp.p, tb, thrust::counting_iterator<uint32_t>(0),
                                        c->rflag.as<uint32_t>(), c->tl.as<uint32_t>(), Lp, (int)tot, st));
    {  // running max of hi along every (slot, segment) row, over the live runs: maxhi[c]
        unsigned long long* sums = c->scan_sums.as<unsigned long long>();
        const unsigned g = (unsigned)std::min<uint64_t>(tot / kScanTile + 1, 148ull * 8);
        (void)launch_chain(pdl, k_segmax_reduce<true>, k_segmax_reduce<false>, g, kScanThreads, 0, st, Lp, n,
                           c->tl.as<uint32_t>(), c->segnum.as<uint32_t>(), c->hi.as<uint32_t>(), sums);
        (void)launch_chain(pdl, k_segmax_tops<true>, k_segmax_tops<false>, 1, 1024, 0, st, Lp, sums);
        (void)launch_chain(pdl, k_segmax_apply<true>, k_segmax_apply<false>, g, kScanThreads, 0, st, Lp, n,
                           c->tl.as<uint32_t>(), c->segnum.as<uint32_t>(), c->hi.as<uint32_t>(), sums,
                           c->maxhi.as<uint32_t>());
        launches += 3;
    }
    // ranges over the live runs, their candidate counts and methods
    const unsigned gc = (unsigned)std::min<uint64_t>(grid_for(tot, 256), (uint64_t)c->num_sms * 32);
    (void)launch_chain(pdl, k_crange_flags<true>, k_crange_flags<false>, gc, 256, 0, st, Lp, n, c->tl.as<uint32_t>(),
                     c->segnum.as<uint32_t>(), c->lo.as<uint32_t>(), c->hi.as<uint32_t>(), c->maxhi.as<uint32_t>(),
                     c->rflag.as<uint32_t>(), c->cl.as<uint64_t>());
    launches++;
    launches += scan_dev(c->scan_sums.as<uint32_t>(), c->rflag.as<uint32_t>(), c->ridx.as<uint32_t>(), Lp, tot, st, pdl);
    launches += scan_dev(c->scan_sums.as<uint64_t>(), c->cl.as<uint64_t>(), c->pc.as<uint64_t>(), Lp, tot, st, pdl);
    (void)launch_chain(pdl, k_crange_emit<true>, k_crange_emit<false>, gc, 256, 0, st, Lp, n, ns, rows, sps,
                     c->tl.as<uint32_t>(), c->seg.as<uint32_t>(), c->segnum.as<uint32_t>(), idx->d_slot,
                     c->lo.as<uint32_t>(), c->maxhi.as<uint32_t>(), c->rflag.as<uint32_t>(), c->ridx.as<uint32_t>(),
                     c->ranges.as<RangeDesc>());
    (void)launch_chain(pdl, k_crange_method<true>, k_crange_method<false>, gc, 256, 0, st, Lp, c->ridx.as<uint32_t>(),
                     c->ranges.as<RangeDesc>(), c->pc.as<uint64_t>(), L.pair_ratio, c->method.as<uint8_t>(),
                     c->rlen.as<uint64_t>(), c->seg_need.as<unsigned long long>(), Rp,
                     reinterpret_cast<unsigned long long*>(d_small + 4));
    launches += 2;
    // side stream: rank tables of the query segments that have a rank-difference range
    RGL_TRY(stream_after(sd, st, c->ev_fork));
    k_seg_tabsize<<<grid_for(n + 1, 256), 256, 0, sd>>>(n, c->segnum.as<uint32_t>(), c->seg_begin.as<uint32_t>(),
                                                        c->seg_need.as<unsigned long long>(), c->ends.as<uint32_t>(),
                                                        c->segtab.as<SegTab>(), c->tab_len.as<uint32_t>());
    tb = c->cub_tmp2.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp2.p, tb, c->tab_len.as<uint32_t>(), c->tab_off.as<uint32_t>(),
                                           (int)n + 1, sd));
    const uint64_t tab_cap = 10ull * n + 16;
    uint32_t* tab_count = d_small + 14;
    k_tab_zero<<<(unsigned)std::min<uint64_t>(grid_for(tab_cap, 256), (uint64_t)c->num_sms * 32), 256, 0, sd>>>(
        n, c->segnum.as<uint32_t>(), c->tab_off.as<uint32_t>(), c->tab_xs.as<uint32_t>(), c->tab_xe.as<uint32_t>(),
        tab_count);
    (void)launch_chain(pdl, k_tab_place<true>, k_tab_place<false>, grid_for(n, 256), 256, 0, sd, n,
                     c->segnum.as<uint32_t>(), c->segtab.as<SegTab>(), c->tab_off.as<uint32_t>(),
                     c->tab_xs.as<uint32_t>(), c->tab_xe.as<uint32_t>());
    (void)launch_chain(pdl, k_tab_count<true>, k_tab_count<false>, grid_for(n, 256), 256, 0, sd, n,
                     c->segnum.as<uint32_t>(), c->segtab.as<SegTab>(), c->starts.as<uint32_t>(),
                     c->ends.as<uint32_t>(), c->tab_xs.as<uint32_t>(), c->tab_xe.as<uint32_t>());
    // inclusive scans written one entry ahead: exclusive scan into tab_* whose entry k + 1 is the
    // inclusive sum through k (the tables are read from tab_* + 1)
    uint32_t* sums2 = c->scan_sums2.as<uint32_t>();
    launches += scan_dev(sums2, c->tab_xs.as<uint32_t>(), c->tab_s.as<uint32_t>(), tab_count, tab_cap, sd, pdl);
    launches += scan_dev(sums2, c->tab_xe.as<uint32_t>(), c->tab_e.as<uint32_t>(), tab_count, tab_cap, sd, pdl);
    (void)launch_chain(pdl, k_tab_interleave<true>, k_tab_interleave<false>,
                     (unsigned)std::min<uint64_t>(grid_for(tab_cap, 256), (uint64_t)c->num_sms * 32), 256, 0, sd,
                     tab_count, c->tab_s.as<uint32_t>(), c->tab_e.as<uint32_t>(), c->tab2.as<uint2>());
    launches++;
    launches += 4;
    // main stream: the pair work space and the rank ranges' positions
    (void)launch_chain(pdl, k_cpair_len<true>, k_cpair_len<false>, gc, 256, 0, st, Lp, n, ns, rows, sps,
                     c->tl.as<uint32_t>(), c->seg.as<uint32_t>(), idx->d_slot, idx->d_layers, c->lo.as<uint32_t>(),
                     c->hi.as<uint32_t>(), c->rflag.as<uint32_t>(), c->ridx.as<uint32_t>(), c->method.as<uint8_t>(),
                     c->starts.as<uint32_t>(), c->val_b.as<uint32_t>(), c->plen.as<uint64_t>(),
                     c->psegs.as<PairSeg>());
    launches++;
    launches += scan_dev(c->scan_sums.as<uint64_t>(), c->rlen.as<uint64_t>(), c->rpos.as<uint64_t>(), Rp, tot, st, pdl);
    launches += scan_dev(c->scan_sums.as<uint64_t>(), c->plen.as<uint64_t>(), c->ppos.as<uint64_t>(), Lp, tot, st, pdl);
    if (mode.no_sweep) {
        k_totals<<<1, 32, 0, st>>>(d_small, c->rpos.as<uint64_t>(), c->ppos.as<uint64_t>());
        launches++;
        RGL_TRY(stream_after(st, sd, c->ev_join));
        c->last_tot = tot;
        c->last_launches = launches;
        c->last_n = n;
        if (mode.reset_err) RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
        return RGL_OK;
    }
    (void)launch_chain(pdl, k_item_ranges<true>, k_item_ranges<false>, (unsigned)(c->num_sms * 8), 256, 0, st,
                     d_small, Rp, c->rpos.as<uint64_t>(), Lp, c->ppos.as<uint64_t>(), L.chunk, kItemCap,
                     c->item_r0.as<uint32_t>(), c->item_t0.as<uint32_t>());
    launches++;
    SweepParams P;
    P.item_r0 = c->item_r0.as<uint32_t>();
    P.item_t0 = c->item_t0.as<uint32_t>();
    P.ppos = c->ppos.as<uint64_t>();
    P.psegs = c->psegs.as<PairSeg>();
    P.segtabs = c->segtab.as<SegTab>();
    P.tab2 = c->tab2.as<uint2>();
    P.item_cap = kItemCap;
    P.rpos = c->rpos.as<uint64_t>();
    P.rcount = Rp;
    P.pcount = Lp;
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
    // tally: one row in a block-wide histogram for the whole kernel (1); several rows in a histogram
    // of each block item's row (2); else (or with RGL_QF_GLOBAL_TALLY) atomics on the outputs (0)
    P.smem_tally = smem > 160 * 1024 ? 0 : rows == 1 ? 1 : (opts && (opts->flags & RGL_QF_GLOBAL_TALLY)) ? 0 : 2;

    if (!P.smem_tally) smem = 0;
    unsigned grid = (unsigned)(c->num_sms * L.ctas_per_sm);
    // the rank tables are joined before the sweeps; the two sweeps run one after the other on
    // `st` (each fills every SM with persistent blocks; run side by side they were slower)
    RGL_TRY(stream_after(st, sd, c->ev_join));
    if (ev) RGL_CUDA(cudaEventRecord(c->ev[1], st));
    if (c->timing && mode.events) RGL_TRY(timing_record(c, true));
    if (P.smem_tally == 2) {
        if (with_bp) k_sweep<true, true><<<grid, 256, smem, st>>>(P);
        else k_sweep<false, true><<<grid, 256, smem, st>>>(P);
    } else {
        if (with_bp) k_sweep<true, false><<<grid, 256, smem, st>>>(P);
        else k_sweep<false, false><<<grid, 256, smem, st>>>(P);
    }
    P.queue = d_small + 2;  // the pair sweep pulls from its own counter
    if (P.smem_tally == 2) {
        if (with_bp) k_pairs<true, true, 1><<<grid, 256, smem, st>>>(P);
        else k_pairs<false, true, 1><<<grid, 256, smem, st>>>(P);
    } else if (P.smem_tally) {
        if (with_bp) k_pairs<true, true, 0><<<grid, 256, smem, st>>>(P);
        else k_pairs<false, true, 0><<<grid, 256, smem, st>>>(P);
    } else {
        if (with_bp) k_pairs<true, false, 0><<<grid, 256, smem, st>>>(P);
        else k_pairs<false, false, 0><<<grid, 256, smem, st>>>(P);
    }
    launches++;
    launches++;
    RGL_CUDA(cudaGetLastError());
    if (c->timing && mode.events) RGL_TRY(timing_record(c, false));
    if (mode.acc) {
        k_acc_stats<<<1, 32, 0, st>>>(mode.acc, d_small + 9, reinterpret_cast<unsigned long long*>(d_small + 4),
                                      reinterpret_cast<unsigned long long*>(d_small + 10),
                                      reinterpret_cast<unsigned long long*>(d_small + 12), n);
        launches++;
    }
    c->last_tot = tot;
    c->last_launches = launches;
    c->last_n = n;
    if (ev) {
        RGL_CUDA(cudaEventRecord(c->ev[2], st));
        RGL_CUDA(cudaMemcpyAsync(c->h_small + 4, d_small + 4, 48, cudaMemcpyDeviceToHost, st));
    }
    if (mode.reset_err) RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
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

// Copies the blocks' host intervals into the context's interval buffer at offsets off, one copy per
// run of blocks that lie back to back in host memory (a file read into one buffer).
int copy_blocks(rgl_context* c, const std::vector<const rgl_query_shard*>& blocks, const std::vector<uint64_t>& off,
                cudaStream_t st) {
    for (size_t i = 0; i < blocks.size();) {
        size_t j = i + 1;
        while (j < blocks.size() && blocks[j]->intervals == blocks[j - 1]->intervals + blocks[j - 1]->count) j++;
        RGL_CUDA(cudaMemcpyAsync(c->iv.as<rgl_interval>() + off[i], blocks[i]->intervals,
                                 (off[j] - off[i]) * sizeof(rgl_interval), cudaMemcpyHostToDevice, st));
        i = j;
    }
    return RGL_OK;
}

// ---- batched form ------------------------------------------------------------------------------
// A batch is cut into sub-batches of at most `sub` intervals (cutting blocks where needed: counts and
// base pairs are sums over pairs, so a row split across sub-batches adds up to the same cells).
struct SubBatch {
    uint64_t begin, n;        // element range in d_intervals
    uint32_t row_lo, rows;    // output rows the sub-batch may touch
    uint32_t tab_at, nblk;    // its block table: entries [tab_at, tab_at + nblk] of the offsets, [tab_at, +nblk) of shards
};

struct BatchPlan {
    std::vector<SubBatch> subs;
    std::vector<uint64_t> off;   // per sub-batch: nblk + 1 offsets relative to its begin
    std::vector<uint32_t> shard; // per sub-batch: nblk shard ids (padded to the offsets' layout)
    std::vector<uint32_t> row;   // per sub-batch: nblk block rows (same layout; unused without block_rows)
    uint64_t max_n = 0;
    uint32_t max_rows = 0, max_blk = 0;
    // per sub-batch: whether the block-local key sort applies, and its shape
    std::vector<char> local;
    std::vector<LocalSort> ls;
    // the sorts' segment-order layouts, in the offsets' (soff, sdst) and shards' (sidx) layouts
    std::vector<uint64_t> soff, sdst;
    std::vector<uint32_t> sidx;
    void prepare(bool block_rows) {
        local.assign(subs.size(), 0);
        ls.assign(subs.size(), LocalSort());
        soff = off;
        sdst = off;
        sidx.assign(shard.size(), 0);
        for (size_t k = 0; k < subs.size(); k++) {
            const SubBatch& sb = subs[k];
            local[k] = blocks_local(sb.nblk, &off[sb.tab_at], &shard[sb.tab_at],
                                    block_rows ? &row[sb.tab_at] : nullptr, sb.rows, sb.row_lo, &ls[k]);
            if (!local[k] || ls[k].dst.empty()) continue;
            std::copy(ls[k].soff.begin(), ls[k].soff.end(), soff.begin() + sb.tab_at);
            std::copy(ls[k].dst.begin(), ls[k].dst.end(), sdst.begin() + sb.tab_at);
            std::copy(ls[k].idx.begin(), ls[k].idx.end(), sidx.begin() + sb.tab_at);
        }
    }
    std::vector<uint64_t> off_table() const {  // the device table: offsets, then soff, then sdst
        std::vector<uint64_t> v(off);
        v.insert(v.end(), soff.begin(), soff.end());
        v.insert(v.end(), sdst.begin(), sdst.end());
        return v;
    }
    std::vector<uint32_t> shard_rows() const {  // the device table: shards, then rows, then sidx
        std::vector<uint32_t> v(shard);
        v.insert(v.end(), row.begin(), row.end());
        v.insert(v.end(), sidx.begin(), sidx.end());
        return v;
    }
    // The pipeline input of sub-batch k over intervals iv, with the device tables d_off / d_sr.
    PipeIn pipe_in(size_t k, const rgl_interval* iv, const uint64_t* d_off, const uint32_t* d_sr,
                   bool block_rows) const {
        const SubBatch& sb = subs[k];
        PipeIn in{iv, sb.n, sb.rows, sb.row_lo, sb.nblk, d_off + sb.tab_at, d_sr + sb.tab_at,
                  block_rows ? d_sr + shard.size() + sb.tab_at : nullptr};
        in.block_local = local[k];
        in.ls.max_block = ls[k].max_block;  // the layout goes by the device tables below
        in.ls.tiles = ls[k].tiles;
        in.ls.chunks = ls[k].chunks;
        if (local[k] && !ls[k].dst.empty()) {
            in.sort_off = d_off + off.size() + sb.tab_at;
            in.sort_dst = d_off + 2 * off.size() + sb.tab_at;
            in.sort_idx = d_sr + 2 * shard.size() + sb.tab_at;
        }
        return in;
    }
};

// Region bits of a sub-batch of `rows` rows under the batch options (0: segments per (shard, row)).
uint32_t batch_region_bits(const rgl_batch_opts* o, uint32_t rows) {
    const uint32_t r = o ? o->region_bits : 0u;
    if (r == RGL_BATCH_NO_REGIONS || r == 0 || rows <= 1) return 0;
    return r;
}

// Region-ordered work needs the device-wide key sort (the block-local sort keeps block order).
void set_regions(PipeIn& in, uint32_t rb) {
    in.region_bits = rb;
    if (rb) in.block_local = 0;
}

int plan_batch(rgl_context* c, const rgl_batch* b, uint64_t sub, BatchPlan* P) {
    const uint64_t* bo = b->block_offsets;
    for (uint32_t i = 0; i < b->num_blocks; i++) {
        if (bo[i + 1] < bo[i]) return fail(RGL_ERR_INVALID_ARGUMENT, "block offsets must be non-decreasing");
        if (b->block_shards[i] >= c->idx->num_shards) return fail(RGL_ERR_INVALID_ARGUMENT, "shard id out of range");
        if (b->block_rows && b->block_rows[i] >= b->num_rows)
            return fail(RGL_ERR_INVALID_ARGUMENT, "block row >= num_rows");
    }
    SubBatch cur{};
    uint32_t rlo = 0xFFFFFFFFu, rhi = 0;
    bool open = false;
    auto close = [&]() {
        if (!open) return;
        P->off.push_back(cur.n);
        P->shard.push_back(0);  // keeps the three tables indexed alike
        P->row.push_back(0);
        cur.row_lo = b->block_rows ? rlo : 0;
        cur.rows = b->block_rows ? rhi - rlo + 1 : b->num_rows;
        P->max_n = std::max(P->max_n, cur.n);
        P->max_rows = std::max(P->max_rows, cur.rows);
        P->max_blk = std::max(P->max_blk, cur.nblk);
        P->subs.push_back(cur);
        open = false;
    };
    for (uint32_t i = 0; i < b->num_blocks; i++) {
        uint64_t at = bo[i], end = bo[i + 1];
        while (at < end) {
            if (!open) {
                cur = SubBatch{at, 0, 0, 0, (uint32_t)P->off.size(), 0};
                rlo = 0xFFFFFFFFu;
                rhi = 0;
                open = true;
            }
            const uint64_t take = std::min(end - at, sub - cur.n);
            P->off.push_back(cur.n);
            P->shard.push_back(b->block_shards[i]);
            P->row.push_back(b->block_rows ? b->block_rows[i] : 0);
            cur.nblk++;
            cur.n += take;
            if (b->block_rows) {
                rlo = std::min(rlo, b->block_rows[i]);
                rhi = std::max(rhi, b->block_rows[i]);
            }
            at += take;
            if (cur.n == sub) close();
        }
    }
    close();
    P->prepare(b->block_rows != nullptr);
    return RGL_OK;
}

Launch batch_launch(rgl_context* c, const rgl_batch_opts* o, rgl_query_opts* q) {
    *q = o ? o->query : rgl_query_opts{};
    if (o && (o->flags & RGL_BF_TUNED) && c->has_tuned) {
        if (!q->chunk) q->chunk = c->tuned.chunk;
        if (!q->ctas_per_sm) q->ctas_per_sm = c->tuned.ctas_per_sm;
        if (!q->pair_ratio) q->pair_ratio = c->tuned.pair_ratio;
    }
    return pick_launch(q);
}

// Enqueues a whole batch on the context stream: zero the outputs, one pipeline run per sub-batch,
// then the error word and the stats accumulator to pinned host memory.
int enqueue_batch(rgl_context* c, const rgl_batch* b, const BatchPlan& P, const uint64_t* d_off,
                  const uint32_t* d_sr, const rgl_query_opts* q, uint32_t* d_counts, unsigned long long* d_bp,
                  bool events, uint32_t* launches, const rgl_batch_opts* o) {
    cudaStream_t st = c->stream;
    const uint32_t D = c->idx->num_sources;
    uint32_t* d_small = c->small.as<uint32_t>();
    RGL_CUDA(cudaMemsetAsync(d_small, 0, 64, st));
    RGL_CUDA(cudaMemsetAsync(c->acc.p, 0, 64, st));
    RGL_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)b->num_rows * D * 4, st));
    if (d_bp) RGL_CUDA(cudaMemsetAsync(d_bp, 0, (size_t)b->num_rows * D * 8, st));
    PipeMode m;
    m.zero_out = false;
    m.reset_err = false;
    m.events = events;
    m.acc = c->acc.as<unsigned long long>();
    uint32_t nl = 0;
    for (size_t k = 0; k < P.subs.size(); k++) {
        const SubBatch& sb = P.subs[k];
        PipeIn in = P.pipe_in(k, b->d_intervals + sb.begin, d_off, d_sr, b->block_rows != nullptr);
        set_regions(in, batch_region_bits(o, sb.rows));
        RGL_TRY(run_pipeline(c, in, q, d_counts + (uint64_t)sb.row_lo * D,
                             d_bp ? d_bp + (uint64_t)sb.row_lo * D : nullptr, nullptr, m));
        nl += c->last_launches;
    }
    RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaMemcpyAsync(c->h_acc, c->acc.p, 64, cudaMemcpyDeviceToHost, st));
    *launches = nl;
    return RGL_OK;
}

void graph_drop(rgl_context* c) {
    if (c->gc.exec) cudaGraphExecDestroy(c->gc.exec);
    if (c->gc.graph) cudaGraphDestroy(c->gc.graph);
    c->gc.exec = nullptr;
    c->gc.graph = nullptr;
    c->gc.key.clear();
}

std::vector<uint64_t> batch_key(rgl_context* c, const rgl_batch* b, const rgl_batch_opts* o, const Launch& L,
                                const void* d_counts, const void* d_bp) {
    std::vector<uint64_t> k;
    k.reserve(16 + 3ull * b->num_blocks);
    k.push_back(b->num_rows);
    k.push_back(b->num_blocks);
    k.push_back((uint64_t)(uintptr_t)b->d_intervals);
    k.push_back((uint64_t)(uintptr_t)d_counts);
    k.push_back((uint64_t)(uintptr_t)d_bp);
    k.push_back(((uint64_t)L.chunk << 32) | L.ctas_per_sm);
    k.push_back(((uint64_t)L.pair_ratio << 32) | (o ? o->query.flags : 0));
    k.push_back(o ? o->sub_batch : 0);
    k.push_back(o ? o->region_bits : 0);
    k.push_back(c->ws_sig);
    k.push_back(b->block_rows ? 1 : 0);
    for (uint32_t i = 0; i <= b->num_blocks; i++) k.push_back(b->block_offsets[i]);
    for (uint32_t i = 0; i < b->num_blocks; i++)
        k.push_back(((uint64_t)b->block_shards[i] << 32) | (b->block_rows ? b->block_rows[i] : 0));
    return k;
}

}  // namespace

namespace rgl {

cudaStream_t context_stream(rgl_context* c) { return c->stream; }

int context_reserve_rows(rgl_context* c, uint64_t max_intervals, uint32_t max_rows, uint32_t max_blocks) {
    RGL_CUDA(cudaSetDevice(c->idx->device));
    return ensure_workspace(c, max_intervals, max_rows, max_blocks);
}

int context_growth_bytes(rgl_context* c, uint64_t n, uint32_t rows, uint32_t nblk, uint64_t* bytes) {
    return size_workspace(c, n, rows, nblk, bytes);
}

// One batch whose intervals are already on the device, rows taken from the blocks (interval sids are
// ignored), as a single pipeline run: zero the num_rows x D outputs, sweep, error word to the host.
// Asynchronous on the context stream; the caller synchronises and then calls context_errors.
int enqueue_block_rows(rgl_context* c, uint32_t num_rows, uint32_t nblk, const uint32_t* shards, const uint32_t* rows,
                       const uint64_t* off, const rgl_interval* d_iv, const rgl_query_opts* q, uint32_t* d_counts,
                       unsigned long long* d_bp) {
    cudaStream_t st = c->stream;
    const uint32_t D = c->idx->num_sources;
    for (uint32_t i = 0; i < nblk; i++)
        if (shards[i] >= c->idx->num_shards || rows[i] >= num_rows)
            return fail(RGL_ERR_INVALID_ARGUMENT, "block shard or row out of range");
    const uint64_t n = nblk ? off[nblk] - off[0] : 0;
    RGL_TRY(ensure_workspace(c, n, 0, nblk));
    std::vector<uint64_t> rel(nblk + 1);
    for (uint32_t i = 0; i <= nblk; i++) rel[i] = off[i] - off[0];
    // device tables: offsets then the sort's segment-order offsets and destinations; shards, rows,
    // then the blocks' ranks in segment order
    LocalSort ls;
    const bool local = blocks_local(nblk, rel.data(), shards, rows, num_rows, 0, &ls);
    const bool perm = local && !ls.dst.empty();
    std::vector<uint64_t> ot(rel);
    if (perm) {
        ot.insert(ot.end(), ls.soff.begin(), ls.soff.end());
        ot.insert(ot.end(), ls.dst.begin(), ls.dst.end());
    }
    std::vector<uint32_t> sr(3ull * nblk + 3, 0);
    for (uint32_t i = 0; i < nblk; i++) {
        sr[i] = shards[i];
        sr[nblk + 1 + i] = rows[i];
        if (perm) sr[2 * (nblk + 1) + i] = ls.idx[i];
    }
    RGL_TRY(c->bt_off.ensure(ot.size() * 8 + 8));
    RGL_TRY(c->bt_shard.ensure(sr.size() * 4 + 4));
    RGL_CUDA(cudaMemcpyAsync(c->bt_off.p, ot.data(), ot.size() * 8, cudaMemcpyHostToDevice, st));
    RGL_CUDA(cudaMemcpyAsync(c->bt_shard.p, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice, st));
    // the interval copies and table uploads above are ordered before the pipeline on this stream
    RGL_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)num_rows * D * 4, st));
    if (d_bp) RGL_CUDA(cudaMemsetAsync(d_bp, 0, (size_t)num_rows * D * 8, st));
    PipeIn in{d_iv + off[0], n, num_rows, 0, nblk, c->bt_off.as<uint64_t>(), c->bt_shard.as<uint32_t>(),
              c->bt_shard.as<uint32_t>() + nblk + 1, 1};
    in.block_local = local;
    if (perm) {
        in.sort_off = c->bt_off.as<uint64_t>() + (nblk + 1);
        in.sort_dst = c->bt_off.as<uint64_t>() + 2 * (nblk + 1);
        in.sort_idx = c->bt_shard.as<uint32_t>() + 2 * (nblk + 1);
    }
    in.ls = std::move(ls);
    PipeMode m;
    m.zero_out = false;
    // the table uploads read pageable vectors that die here: an asynchronous copy from pageable
    // memory has staged its source before it returns
    return run_pipeline(c, in, q, d_counts, d_bp, nullptr, m);
}

// After the stream has been synchronised: the error bits of the last run.
int context_errors(rgl_context* c) { return finish(c, pick_launch(nullptr), nullptr); }

uint32_t context_last_launches(rgl_context* c) { return c->last_launches; }

}  // namespace rgl

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
    if (s == RGL_OK && (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
                        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess))
        s = fail(RGL_ERR_DEVICE, "side stream");
    if (s == RGL_OK) cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, index->device);
    // shared-memory tallies of up to 160 KB (one row, D x 12 B); set once here so that no launch
    // path changes function attributes (graph capture included)
    if (s == RGL_OK) {
        const int mx = 160 * 1024;
        if (cudaFuncSetAttribute(k_sweep<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess ||
            cudaFuncSetAttribute(k_sweep<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess ||
            cudaFuncSetAttribute(k_sweep<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess ||
            cudaFuncSetAttribute(k_sweep<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) != cudaSuccess ||
            cudaFuncSetAttribute(k_pairs<true, true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_pairs<false, true, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_pairs<true, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_pairs<false, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx) !=
                cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "cudaFuncSetAttribute");
    }
    for (int i = 0; i < 4 && s == RGL_OK; i++)
        if (cudaEventCreate(&c->ev[i]) != cudaSuccess) s = fail(RGL_ERR_DEVICE, "cudaEventCreate");
    if (s == RGL_OK && cudaMallocHost(&c->h_small, 256) != cudaSuccess) s = fail(RGL_ERR_OOM, "pinned");
    if (s == RGL_OK && cudaMallocHost(&c->h_acc, 64) != cudaSuccess) s = fail(RGL_ERR_OOM, "pinned");
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
    if (c->side) cudaStreamSynchronize(c->side);
    DevBuf* bufs[] = {&c->iv, &c->blk_off, &c->blk_shard, &c->key_a, &c->key_b, &c->val_a, &c->val_b,
                      &c->ekey_a, &c->ekey_b, &c->starts, &c->ends, &c->seg, &c->segflag, &c->segnum,
                      &c->seg_begin, &c->ps_in, &c->pe_in, &c->ps, &c->pe, &c->lo, &c->hi, &c->maxhi,
                      &c->rflag, &c->ridx, &c->ranges, &c->rlen, &c->rpos, &c->cub_tmp, &c->small,
                      &c->out_counts, &c->out_bp, &c->item_r0,
                      &c->segtab, &c->tab_len, &c->tab_off, &c->tab_s, &c->tab_e, &c->tab_xs, &c->tab_xe, &c->tab2,
                      &c->cl, &c->pc, &c->method, &c->tl, &c->scan_sums, &c->plen, &c->ppos, &c->psegs, &c->item_t0,
                      &c->seg_need, &c->item_hits, &c->item_base, &c->pairs, &c->bt_off, &c->bt_shard, &c->acc, &c->gc.t_off, &c->gc.t_shard,
                      &c->cub_tmp2, &c->scan_sums2, &c->sortplan, &c->sort_tab, &c->sort_rank};
    if (c->gc.exec) cudaGraphExecDestroy(c->gc.exec);
    if (c->gc.graph) cudaGraphDestroy(c->gc.graph);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    for (DevBuf* b : bufs) b->release();
    for (int i = 0; i < 2; i++) {
        c->stage[i].release();
        if (c->ev_copied[i]) cudaEventDestroy(c->ev_copied[i]);
        if (c->ev_used[i]) cudaEventDestroy(c->ev_used[i]);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->tev) cudaEventDestroy(e);
    if (c->h_small) cudaFreeHost(c->h_small);
    if (c->h_acc) cudaFreeHost(c->h_acc);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
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
    PipeIn in{c->iv.as<rgl_interval>(), n, num_rows, 0, num_shards, c->blk_off.as<uint64_t>(),
              c->blk_shard.as<uint32_t>(), nullptr};
    in.block_local = blocks_local(num_shards, off.data(), shard_ids, nullptr, num_rows, 0, &in.ls);
    RGL_TRY(run_pipeline(c, in, opts, d_counts, reinterpret_cast<unsigned long long*>(d_overlap_bp), stats));
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
    RGL_TRY(copy_blocks(c, blocks, off, st));
    if (!blocks.empty()) {
        RGL_CUDA(cudaMemcpyAsync(c->blk_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st));
        RGL_CUDA(cudaMemcpyAsync(c->blk_shard.p, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, st));
    }
    PipeIn in{c->iv.as<rgl_interval>(), n, rows, 0, (uint32_t)blocks.size(), c->blk_off.as<uint64_t>(),
              c->blk_shard.as<uint32_t>(), nullptr};
    in.block_local = blocks_local((uint32_t)blocks.size(), off.data(), ids.data(), nullptr, rows, 0, &in.ls);
    RGL_TRY(run_pipeline(c, in, opts, c->out_counts.as<uint32_t>(),
                         overlap_bp ? c->out_bp.as<unsigned long long>() : nullptr, stats));
    if (cells) {
        RGL_CUDA(cudaMemcpyAsync(counts, c->out_counts.p, cells * 4, cudaMemcpyDeviceToHost, st));
        if (overlap_bp) RGL_CUDA(cudaMemcpyAsync(overlap_bp, c->out_bp.p, cells * 8, cudaMemcpyDeviceToHost, st));
    }
    RGL_CUDA(cudaStreamSynchronize(st));
    return finish(c, pick_launch(opts), stats);
}

int rgl_query_batch_device(rgl_context* c, const rgl_batch* b, const rgl_batch_opts* o, uint32_t* d_counts,
                           uint64_t* d_overlap_bp, rgl_batch_stats* stats) {
    clear_error();
    if (!c || !b || !d_counts) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    if (b->num_blocks && (!b->block_offsets || !b->block_shards || !b->d_intervals))
        return fail(RGL_ERR_INVALID_ARGUMENT, "incomplete batch");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    const uint64_t sub = (o && o->sub_batch) ? std::min<uint64_t>(o->sub_batch, kMaxRunIntervals) : (1ull << 25);
    rgl_query_opts q;
    const Launch L = batch_launch(c, o, &q);
    const bool graph = o && (o->flags & RGL_BF_GRAPH);
    unsigned long long* d_bp = (d_overlap_bp && !(q.flags & RGL_QF_NO_OVERLAP))
                                   ? reinterpret_cast<unsigned long long*>(d_overlap_bp) : nullptr;
    cudaStream_t st = c->stream;
    BatchPlan P;
    std::vector<uint64_t> key;
    bool replay = false;
    if (graph) {
        key = batch_key(c, b, o, L, d_counts, d_bp);
        replay = c->gc.exec && key == c->gc.key;
    }
    if (!replay) {
        RGL_TRY(plan_batch(c, b, sub, &P));
        RGL_TRY(ensure_workspace(c, P.max_n, 0, P.max_blk));
    }
    if (stats) RGL_CUDA(cudaEventRecord(c->ev[0], st));
    uint32_t launches = 0, subs = 0, nodes = 0;
    if (replay) {
        RGL_CUDA(cudaGraphLaunch(c->gc.exec, st));
        launches = c->gc.launches;
        subs = c->gc.subs;
        nodes = c->gc.nodes;
    } else if (graph) {
        RGL_CUDA(cudaStreamSynchronize(st));  // the previous graph may still read its tables
        graph_drop(c);
        const std::vector<uint64_t> ot = P.off_table();
        RGL_TRY(c->gc.t_off.ensure(ot.size() * 8 + 8));
        const std::vector<uint32_t> sr = P.shard_rows();
        RGL_TRY(c->gc.t_shard.ensure(sr.size() * 4 + 4));
        RGL_CUDA(cudaMemcpy(c->gc.t_off.p, ot.data(), ot.size() * 8, cudaMemcpyHostToDevice));
        RGL_CUDA(cudaMemcpy(c->gc.t_shard.p, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice));
        // the key is taken after the workspace is sized, so that a later reallocation invalidates it
        key = batch_key(c, b, o, L, d_counts, d_bp);
        RGL_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int s = enqueue_batch(c, b, P, c->gc.t_off.as<uint64_t>(), c->gc.t_shard.as<uint32_t>(), &q, d_counts, d_bp,
                              false, &launches, o);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s != RGL_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return fail(RGL_ERR_DEVICE, std::string("stream capture: ") + cudaGetErrorString(e));
        cudaGraphExec_t x = nullptr;
        e = cudaGraphInstantiate(&x, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return fail(RGL_ERR_DEVICE, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        c->gc.graph = g;
        c->gc.exec = x;
        c->gc.key = std::move(key);
        c->gc.nodes = nodes = (uint32_t)nn;
        c->gc.launches = launches;
        c->gc.subs = subs = (uint32_t)P.subs.size();
        RGL_CUDA(cudaGraphLaunch(x, st));
    } else {
        const std::vector<uint64_t> ot = P.off_table();
        RGL_TRY(c->bt_off.ensure(ot.size() * 8 + 8));
        const std::vector<uint32_t> sr = P.shard_rows();
        RGL_TRY(c->bt_shard.ensure(sr.size() * 4 + 4));
        RGL_CUDA(cudaMemcpyAsync(c->bt_off.p, ot.data(), ot.size() * 8, cudaMemcpyHostToDevice, st));
        RGL_CUDA(cudaMemcpyAsync(c->bt_shard.p, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice, st));
        RGL_TRY(enqueue_batch(c, b, P, c->bt_off.as<uint64_t>(), c->bt_shard.as<uint32_t>(), &q, d_counts, d_bp, true,
                              &launches, o));
        subs = (uint32_t)P.subs.size();
    }
    c->last_n = 0;  // the single-call stats of finish() do not apply to a batch
    if (!stats) return RGL_OK;
    RGL_CUDA(cudaEventRecord(c->ev[2], st));
    RGL_CUDA(cudaStreamSynchronize(st));
    float ms = 0;
    RGL_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[2]));
    std::memset(stats, 0, sizeof(*stats));
    stats->ranges = c->h_acc[0];
    stats->db_swept = c->h_acc[1];
    stats->rank_positions = c->h_acc[2];
    stats->pair_candidates = c->h_acc[3];
    stats->query_intervals = c->h_acc[4];
    stats->sub_batches = subs;
    stats->kernel_launches = launches;
    stats->graph_nodes = nodes;
    stats->graph_replayed = replay ? 1 : 0;
    stats->device_ms = ms;
    stats->chunk = L.chunk;
    stats->ctas_per_sm = L.ctas_per_sm;
    stats->pair_ratio = L.pair_ratio;
    return finish(c, L, nullptr);
}

int rgl_query_batch_host(rgl_context* c, const rgl_batch* b, const rgl_interval* h_intervals, const rgl_batch_opts* o,
                    uint32_t* counts, uint64_t* overlap_bp, rgl_batch_stats* stats) {
    clear_error();
    if (!c || !b || !counts) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    if (b->num_blocks && (!b->block_offsets || !b->block_shards || !h_intervals))
        return fail(RGL_ERR_INVALID_ARGUMENT, "incomplete batch");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    const uint64_t sub = (o && o->sub_batch) ? std::min<uint64_t>(o->sub_batch, kMaxRunIntervals) : (1ull << 25);
    rgl_query_opts q;
    const Launch L = batch_launch(c, o, &q);
    const bool want_bp = overlap_bp && !(q.flags & RGL_QF_NO_OVERLAP);
    const uint32_t D = c->idx->num_sources;
    const uint64_t cells = (uint64_t)b->num_rows * D;
    BatchPlan P;
    RGL_TRY(plan_batch(c, b, sub, &P));
    RGL_TRY(ensure_workspace(c, P.max_n, b->num_rows, P.max_blk));
    for (int i = 0; i < 2; i++) {
        RGL_TRY(c->stage[i].ensure(std::max<uint64_t>(P.max_n, 1) * sizeof(rgl_interval)));
        if (!c->ev_copied[i]) RGL_CUDA(cudaEventCreateWithFlags(&c->ev_copied[i], cudaEventDisableTiming));
        if (!c->ev_used[i]) RGL_CUDA(cudaEventCreateWithFlags(&c->ev_used[i], cudaEventDisableTiming));
    }
    if (!c->copy_stream) RGL_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    cudaStream_t st = c->stream, cs = c->copy_stream;
    const std::vector<uint32_t> sr = P.shard_rows();
    const std::vector<uint64_t> ot = P.off_table();
    RGL_TRY(c->bt_off.ensure(ot.size() * 8 + 8));
    RGL_TRY(c->bt_shard.ensure(sr.size() * 4 + 4));
    if (stats) RGL_CUDA(cudaEventRecord(c->ev[0], st));
    RGL_CUDA(cudaMemcpyAsync(c->bt_off.p, ot.data(), ot.size() * 8, cudaMemcpyHostToDevice, st));
    RGL_CUDA(cudaMemcpyAsync(c->bt_shard.p, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice, st));
    uint32_t* d_counts = c->out_counts.as<uint32_t>();
    unsigned long long* d_bp = want_bp ? c->out_bp.as<unsigned long long>() : nullptr;
    uint32_t* d_small = c->small.as<uint32_t>();
    RGL_CUDA(cudaMemsetAsync(d_small, 0, 64, st));
    RGL_CUDA(cudaMemsetAsync(c->acc.p, 0, 64, st));
    RGL_CUDA(cudaMemsetAsync(d_counts, 0, cells * 4, st));
    if (d_bp) RGL_CUDA(cudaMemsetAsync(d_bp, 0, cells * 8, st));
    PipeMode m;
    m.zero_out = false;
    m.reset_err = false;
    m.acc = c->acc.as<unsigned long long>();
    uint32_t launches = 0;
    const uint64_t* d_off = c->bt_off.as<uint64_t>();
    const uint32_t* d_sr = c->bt_shard.as<uint32_t>();
    for (size_t k = 0; k < P.subs.size(); k++) {
        const SubBatch& sb = P.subs[k];
        const int slot = (int)(k & 1);
        rgl_interval* stage = c->stage[slot].as<rgl_interval>();
        // the staging buffer is free once the sub-batch two back has been swept
        if (k >= 2) RGL_CUDA(cudaStreamWaitEvent(cs, c->ev_used[slot], 0));
        RGL_CUDA(cudaMemcpyAsync(stage, h_intervals + sb.begin, sb.n * sizeof(rgl_interval), cudaMemcpyHostToDevice, cs));
        RGL_CUDA(cudaEventRecord(c->ev_copied[slot], cs));
        RGL_CUDA(cudaStreamWaitEvent(st, c->ev_copied[slot], 0));
        PipeIn in = P.pipe_in(k, stage, d_off, d_sr, b->block_rows != nullptr);
        set_regions(in, batch_region_bits(o, sb.rows));
        RGL_TRY(run_pipeline(c, in, &q, d_counts + (uint64_t)sb.row_lo * D, d_bp ? d_bp + (uint64_t)sb.row_lo * D : nullptr,
                             nullptr, m));
        RGL_CUDA(cudaEventRecord(c->ev_used[slot], st));
        launches += c->last_launches;
    }
    RGL_CUDA(cudaMemcpyAsync(c->h_small, d_small, 4, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaMemcpyAsync(c->h_acc, c->acc.p, 64, cudaMemcpyDeviceToHost, st));
    if (cells) {
        RGL_CUDA(cudaMemcpyAsync(counts, d_counts, cells * 4, cudaMemcpyDeviceToHost, st));
        if (overlap_bp) {
            if (d_bp) RGL_CUDA(cudaMemcpyAsync(overlap_bp, d_bp, cells * 8, cudaMemcpyDeviceToHost, st));
            else std::memset(overlap_bp, 0, cells * 8);
        }
    }
    if (stats) RGL_CUDA(cudaEventRecord(c->ev[2], st));
    RGL_CUDA(cudaStreamSynchronize(st));
    c->last_n = 0;
    if (stats) {
        float ms = 0;
        RGL_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[2]));
        std::memset(stats, 0, sizeof(*stats));
        stats->ranges = c->h_acc[0];
        stats->db_swept = c->h_acc[1];
        stats->rank_positions = c->h_acc[2];
        stats->pair_candidates = c->h_acc[3];
        stats->query_intervals = c->h_acc[4];
        stats->sub_batches = (uint32_t)P.subs.size();
        stats->kernel_launches = launches;
        stats->device_ms = ms;
        stats->chunk = L.chunk;
        stats->ctas_per_sm = L.ctas_per_sm;
        stats->pair_ratio = L.pair_ratio;
    }
    return finish(c, L, nullptr);
}

// Autotuner: times the sweep kernels of the batch's largest sub-batch over a grid of launch shapes
// (pair_ratio first at the default shape, then work-item size x CTAs per SM) and keeps the fastest.
int rgl_batch_autotune(rgl_context* c, const rgl_batch* b, uint64_t sub_batch, rgl_query_opts* best,
                       rgl_tune_trial* trials, uint32_t max_trials, uint32_t* num_trials) {
    clear_error();
    if (!c || !b || !best) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    BatchPlan P;
    const uint64_t sub = sub_batch ? std::min<uint64_t>(sub_batch, kMaxRunIntervals) : (1ull << 25);
    RGL_TRY(plan_batch(c, b, sub, &P));
    if (P.subs.empty()) return fail(RGL_ERR_INVALID_ARGUMENT, "empty batch");
    size_t big = 0;
    for (size_t i = 1; i < P.subs.size(); i++)
        if (P.subs[i].n > P.subs[big].n) big = i;
    const SubBatch sb = P.subs[big];
    RGL_TRY(ensure_workspace(c, sb.n, sb.rows, sb.nblk));
    cudaStream_t st = c->stream;
    const std::vector<uint64_t> ot = P.off_table();
    RGL_TRY(c->bt_off.ensure(ot.size() * 8 + 8));
    const std::vector<uint32_t> sr = P.shard_rows();
    RGL_TRY(c->bt_shard.ensure(sr.size() * 4 + 4));
    RGL_CUDA(cudaMemcpyAsync(c->bt_off.p, ot.data(), ot.size() * 8, cudaMemcpyHostToDevice, st));
    RGL_CUDA(cudaMemcpyAsync(c->bt_shard.p, sr.data(), sr.size() * 4, cudaMemcpyHostToDevice, st));
    PipeIn in = P.pipe_in(big, b->d_intervals + sb.begin, c->bt_off.as<uint64_t>(), c->bt_shard.as<uint32_t>(),
                          b->block_rows != nullptr);
    set_regions(in, batch_region_bits(nullptr, sb.rows));
    const bool was_timing = c->timing;
    *best = rgl_query_opts{};
    uint32_t nt = 0;
    auto trial = [&](rgl_query_opts q, float* out_ms) -> int {
        float best_ms = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            c->timing = true;
            c->tev_used = 0;
            RGL_TRY(run_pipeline(c, in, &q, c->out_counts.as<uint32_t>(), c->out_bp.as<unsigned long long>(), nullptr));
            RGL_CUDA(cudaStreamSynchronize(st));
            float ms = 0;
            RGL_CUDA(cudaEventElapsedTime(&ms, c->tev[0], c->tev[1]));
            c->tev_used = 0;
            best_ms = std::min(best_ms, ms);
        }
        *out_ms = best_ms;
        const Launch L = pick_launch(&q);
        if (trials && nt < max_trials) trials[nt] = rgl_tune_trial{L.chunk, L.ctas_per_sm, L.pair_ratio, best_ms};
        nt++;
        return RGL_OK;
    };
    int s = RGL_OK;
    rgl_query_opts cur{};
    cur.flags = 0;
    float cur_ms = 1e30f;
    for (uint32_t pr : {1u, 2u, 4u, 8u}) {
        rgl_query_opts q = cur;
        q.pair_ratio = pr;
        float ms;
        if ((s = trial(q, &ms)) != RGL_OK) break;
        if (ms < cur_ms) {
            cur_ms = ms;
            best->pair_ratio = pr;
        }
    }
    cur.pair_ratio = best->pair_ratio;
    for (uint32_t ch : {512u, 1024u, 2048u, 4096u, 8192u}) {
        if (s != RGL_OK) break;
        for (uint32_t ct : {2u, 3u, 4u, 6u, 8u}) {
            rgl_query_opts q = cur;
            q.chunk = ch;
            q.ctas_per_sm = ct;
            float ms;
            if ((s = trial(q, &ms)) != RGL_OK) break;
            if (ms < cur_ms) {
                cur_ms = ms;
                best->chunk = ch;
                best->ctas_per_sm = ct;
            }
        }
    }
    c->timing = was_timing;
    if (s != RGL_OK) return s;
    const Launch L = pick_launch(best);
    best->chunk = L.chunk;
    best->ctas_per_sm = L.ctas_per_sm;
    best->pair_ratio = L.pair_ratio;
    best->block = 256;
    best->flags = 0;
    c->tuned = *best;
    c->has_tuned = true;
    if (num_trials) *num_trials = nt;
    RGL_CUDA(cudaStreamSynchronize(st));
    return finish(c, L, nullptr);
}

int rgl_query_pairs(rgl_context* c, const rgl_query_batch* b, uint64_t capacity, rgl_pair* pairs,
                    uint64_t* out_count) {
    clear_error();
    if (!c || !b || !out_count) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    RGL_CUDA(cudaSetDevice(c->idx->device));
    *out_count = 0;
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
    RGL_TRY(ensure_workspace(c, n, 0, (uint32_t)blocks.size()));
    cudaStream_t st = c->stream;
    RGL_TRY(copy_blocks(c, blocks, off, st));
    if (!blocks.empty()) {
        RGL_CUDA(cudaMemcpyAsync(c->blk_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st));
        RGL_CUDA(cudaMemcpyAsync(c->blk_shard.p, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, st));
    }
    // every candidate run becomes a pair run: a range is swept pair by pair when its candidates are
    // at most pair_ratio x its union, which no range exceeds at this ratio
    rgl_query_opts q{};
    q.pair_ratio = 0xFFFFFFFFu;
    PipeIn in{c->iv.as<rgl_interval>(), n, b->num_rows, 0, (uint32_t)blocks.size(), c->blk_off.as<uint64_t>(),
              c->blk_shard.as<uint32_t>(), nullptr};
    in.block_local = blocks_local((uint32_t)blocks.size(), off.data(), ids.data(), nullptr, b->num_rows, 0, &in.ls);
    PipeMode m;
    m.zero_out = false;
    m.no_sweep = true;
    RGL_TRY(run_pipeline(c, in, &q, nullptr, nullptr, nullptr, m));
    RGL_CUDA(cudaStreamSynchronize(st));
    RGL_TRY(finish(c, pick_launch(&q), nullptr));
    if (!n || !c->idx->num_slots) return RGL_OK;
    uint64_t positions = 0;  // the pair work space total, small[12..13]
    RGL_CUDA(cudaMemcpy(&positions, c->small.as<uint32_t>() + 12, 8, cudaMemcpyDeviceToHost));
    const uint32_t* Lp = c->small.as<uint32_t>() + 8;
    const uint32_t chunk = 2048;
    const uint64_t items = (positions + chunk - 1) / chunk;
    if (!items) return RGL_OK;
    RGL_TRY(c->item_hits.ensure((items + 1) * 8));
    RGL_TRY(c->item_base.ensure((items + 1) * 8));
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (uint64_t*)nullptr, (uint64_t*)nullptr, (int)(items + 1), st);
    RGL_TRY(c->cub_tmp.ensure(tb + 256));
    const unsigned grid = (unsigned)std::min<uint64_t>((items * 32 + 255) / 256, (uint64_t)c->num_sms * 16);
    RGL_CUDA(cudaMemsetAsync(c->item_hits.as<uint64_t>() + items, 0, 8, st));
    k_pair_list<false><<<grid, 256, 0, st>>>(c->ppos.as<uint64_t>(), Lp, c->psegs.as<PairSeg>(), c->idx->d_pos,
                                             c->idx->d_sid, items, chunk, c->item_hits.as<uint64_t>(), nullptr,
                                             nullptr);
    tb = c->cub_tmp.cap;
    RGL_CUDA(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tb, c->item_hits.as<uint64_t>(), c->item_base.as<uint64_t>(),
                                           (int)(items + 1), st));
    uint64_t hits = 0;
    RGL_CUDA(cudaMemcpyAsync(&hits, c->item_base.as<uint64_t>() + items, 8, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    *out_count = hits;
    if (!pairs || !hits) return RGL_OK;
    if (capacity < hits) return fail(RGL_ERR_INVALID_ARGUMENT, "pair capacity too small (needs " + std::to_string(hits) + ")");
    RGL_TRY(c->pairs.ensure(hits * sizeof(rgl_pair)));
    k_pair_list<true><<<grid, 256, 0, st>>>(c->ppos.as<uint64_t>(), Lp, c->psegs.as<PairSeg>(), c->idx->d_pos,
                                            c->idx->d_sid, items, chunk, nullptr, c->item_base.as<uint64_t>(),
                                            c->pairs.as<rgl_pair>());
    RGL_CUDA(cudaGetLastError());
    RGL_CUDA(cudaMemcpyAsync(pairs, c->pairs.p, hits * sizeof(rgl_pair), cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    return RGL_OK;
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
