// The block-local sort's kernels (its shape and launcher are declared in block_sort.cuh).
#include <cub/block/block_radix_sort.cuh>

#include <type_traits>

#include "block_sort.cuh"

namespace rgl {
namespace {

// The block b with pre[b] <= x < pre[b + 1] (pre: nblk + 1 non-decreasing prefix counts, x < pre[nblk]).
__device__ inline uint32_t find_block(const uint32_t* __restrict__ pre, uint32_t nblk, uint32_t x) {
    uint32_t lo = 0, hi = nblk;
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (__ldg(pre + m) <= x) lo = m; else hi = m;
    }
    return lo;
}

// Exclusive prefix counts of the blocks' tiles and merge chunks, by one thread block: each thread
// sums a contiguous stretch of blocks, a block scan of the stretch totals gives each stretch its
// offset, and the stretch is written.
__global__ void __launch_bounds__(1024) k_sort_plan(uint32_t nblk, const uint64_t* __restrict__ blk_off,
                                                    uint32_t* __restrict__ tile_pre, uint32_t* __restrict__ chunk_pre) {
    __shared__ uint32_t pt[1024], pc[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (nblk + 1023) / 1024;
    const uint32_t a = min(t * per, nblk), b = min(a + per, nblk);
    uint32_t st = 0, sc = 0;
    for (uint32_t i = a; i < b; i++) {
        const uint64_t cnt = blk_off[i + 1] - blk_off[i];
        st += sort_tiles(cnt);
        sc += merge_chunks(cnt);
    }
    pt[t] = st;
    pc[t] = sc;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan of the totals
        const uint32_t vt = t >= off ? pt[t - off] : 0u, vc = t >= off ? pc[t - off] : 0u;
        __syncthreads();
        pt[t] += vt;
        pc[t] += vc;
        __syncthreads();
    }
    uint32_t rt = t ? pt[t - 1] : 0u, rc = t ? pc[t - 1] : 0u;
    for (uint32_t i = a; i < b; i++) {
        tile_pre[i] = rt;
        chunk_pre[i] = rc;
        const uint64_t cnt = blk_off[i + 1] - blk_off[i];
        rt += sort_tiles(cnt);
        rc += merge_chunks(cnt);
    }
    if (t == 1023) {
        tile_pre[nblk] = pt[1023];
        chunk_pre[nblk] = pc[1023];
    }
}

template <bool VALUES>
struct BlockSortTypes {
    using Sort = cub::BlockRadixSort<uint32_t, kBsThreads, kBsItems, typename std::conditional<VALUES, uint32_t, cub::NullType>::type>;
    union Smem {
        typename Sort::TempStorage sort;
        uint32_t last[kBsThreads];
    };
};

// The tiles of ordered blocks, copied to the output (one tile per thread block, coalesced; the
// tiles of other blocks return at once).  Few registers, so the copy runs at full occupancy instead
// of in the sort's register-heavy blocks.
template <bool VALUES>
__global__ void __launch_bounds__(kBsThreads) k_tile_copy(uint32_t nblk, const uint64_t* __restrict__ blk_off,
                                                            const uint32_t* __restrict__ tile_pre,
                                                            const uint32_t* __restrict__ unsorted,
                                                            const uint64_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
                                                            uint32_t* __restrict__ vout) {
    const uint32_t tile = blockIdx.x;
    if (tile >= __ldg(tile_pre + nblk)) return;
    const uint32_t blk = find_block(tile_pre, nblk, tile);
    if (unsorted[blk] != 0u) return;
    const uint64_t bbeg = blk_off[blk], bend = blk_off[blk + 1];
    const uint64_t base = bbeg + (uint64_t)(tile - tile_pre[blk]) * kBlockSortCap;
    const uint64_t rest = bend - base;
    const uint32_t cnt = (uint32_t)(rest < kBlockSortCap ? rest : kBlockSortCap);
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < cnt; i += kBsThreads) {
        kout[base + i] = kin[base + i];
        if (VALUES) vout[base + i] = vin[base + i];
    }
}

// One tile per thread block (grid: an upper bound of the tiles; CTAs past the last tile return).
// With VALUES the start keys with their ends as values (key_a / val_a), else the end keys alone.
// unsorted[b] != 0: block b is not in order (only such blocks are sorted here).  Output: `out` when
// the block needs an even number of merge passes, else in place (`in`); *maxp: the most merge
// passes any of these blocks needs.
template <bool VALUES>
__global__ void __launch_bounds__(kBsThreads) k_tile_sort(uint32_t nblk, const uint64_t* __restrict__ blk_off,
                                                            const uint32_t* __restrict__ tile_pre,
                                                            const uint32_t* __restrict__ unsorted, uint64_t* kin,
                                                            uint32_t* vin, uint64_t* __restrict__ kout,
                                                            uint32_t* __restrict__ vout, uint32_t* __restrict__ maxp) {
    using T = BlockSortTypes<VALUES>;
    extern __shared__ __align__(16) unsigned char bs_smem[];
    typename T::Smem& sm = *reinterpret_cast<typename T::Smem*>(bs_smem);
    const uint32_t tile = blockIdx.x;
    if (tile >= __ldg(tile_pre + nblk)) return;
    const uint32_t blk = find_block(tile_pre, nblk, tile);
    const uint64_t bbeg = blk_off[blk], bcnt = blk_off[blk + 1] - bbeg;
    const uint64_t base = bbeg + (uint64_t)(tile - tile_pre[blk]) * kBlockSortCap;
    const uint64_t rest = bbeg + bcnt - base;
    const uint32_t cnt = (uint32_t)(rest < kBlockSortCap ? rest : kBlockSortCap);
    if (unsorted[blk] == 0u) return;  // an ordered block is copied by k_tile_copy
    const uint32_t passes = sort_passes(bcnt);
    if (threadIdx.x == 0 && tile == tile_pre[blk] && passes) atomicMax(maxp, passes);
    uint64_t* ko = (passes & 1u) ? kin : kout;
    uint32_t* vo = (passes & 1u) ? vin : vout;
    const uint64_t hi = kin[base] & 0xFFFFFFFF00000000ull;  // the block's segment, in the high word
    uint32_t k[kBsItems], v[kBsItems];
    uint32_t any = 0;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < kBsItems; j++) {
        const uint32_t i = threadIdx.x * kBsItems + j;  // blocked: thread t holds [16 t, 16 t + 16)
        k[j] = i < cnt ? (uint32_t)kin[base + i] : 0xFFFFFFFFu;  // padding sorts last
        v[j] = (VALUES && i < cnt) ? vin[base + i] : 0u;
        any |= i < cnt ? k[j] : 0u;
        if (j) ok = ok && k[j - 1] <= k[j];
    }
    __shared__ uint32_t s_bits;  // bitwise OR of the tile's keys
    sm.last[threadIdx.x] = k[kBsItems - 1];
    if (threadIdx.x == 0) s_bits = 0;
    __syncthreads();
    if (threadIdx.x) ok = ok && sm.last[threadIdx.x - 1] <= k[0];
    any = __reduce_or_sync(0xffffffffu, any);
    if ((threadIdx.x & 31u) == 0) atomicOr(&s_bits, any);
    // also orders every read of the tile before the in-place writes below, and the atomicOr
    // before the read of s_bits
    const bool sorted = __syncthreads_and(ok);
    const uint32_t bits = s_bits;
    if (!sorted) {
        const int end_bit = bits ? 32 - __clz(bits) : 1;
        if constexpr (VALUES)
            typename T::Sort(sm.sort).Sort(k, v, 0, end_bit);
        else
            typename T::Sort(sm.sort).Sort(k, 0, end_bit);
    }
#pragma unroll
    for (int j = 0; j < kBsItems; j++) {
        const uint32_t i = threadIdx.x * kBsItems + j;
        if (i < cnt) {
            ko[base + i] = hi | k[j];
            if (VALUES) vo[base + i] = v[j];
        }
    }
}

template <bool VALUES>
constexpr size_t block_sort_smem() { return sizeof(typename BlockSortTypes<VALUES>::Smem); }

// Merge-path split of output diagonal d of runs a (na keys) and b (nb keys): the number of the d
// first outputs that come from a, ties going to a (stability).
template <class K>
__device__ inline uint32_t merge_split(const K* a, uint32_t na, const K* b, uint32_t nb, uint32_t d) {
    uint32_t lo = d > nb ? d - nb : 0u, hi = min(d, na);
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if ((uint32_t)a[m] <= (uint32_t)b[d - 1 - m]) lo = m + 1; else hi = m;
    }
    return lo;
}

// Merge pass q (1-based) of the block sort: one CTA per merge chunk (grid: an upper bound of the
// chunks; CTAs past the last chunk, of ordered blocks or of blocks needing fewer passes return).
// A block needing p passes reads buffer A at pass q when p - q + 1 is odd, else B, and writes the
// other one.
template <bool VALUES>
__global__ void __launch_bounds__(kMergeThreads) k_merge_pass(uint32_t q, uint32_t nblk,
                                                              const uint64_t* __restrict__ blk_off,
                                                              const uint32_t* __restrict__ chunk_pre,
                                                              const uint32_t* __restrict__ unsorted, uint64_t* ka,
                                                              uint32_t* va, uint64_t* kb, uint32_t* vb,
                                                              const uint32_t* __restrict__ maxp) {
    __shared__ uint32_t sk[kMergeChunk], sv[VALUES ? kMergeChunk : 1];
    __shared__ uint32_t ok[kMergeChunk], ov[VALUES ? kMergeChunk : 1];
    __shared__ uint32_t s_split[2];
    if (q > *maxp) return;  // no block out of order needs this pass
    const uint32_t chunk = blockIdx.x;
    if (chunk >= __ldg(chunk_pre + nblk)) return;
    const uint32_t blk = find_block(chunk_pre, nblk, chunk);
    if (unsorted[blk] == 0u) return;
    const uint64_t bbeg = blk_off[blk];
    const uint32_t cnt = (uint32_t)(blk_off[blk + 1] - bbeg);
    const uint32_t p = sort_passes(cnt);
    if (p < q) return;
    const bool from_a = ((p - q + 1) & 1u) != 0u;
    const uint64_t* ks = (from_a ? ka : kb) + bbeg;
    const uint32_t* vs = (from_a ? va : vb) + bbeg;
    uint64_t* kd = (from_a ? kb : ka) + bbeg;
    uint32_t* vd = (from_a ? vb : va) + bbeg;
    const uint32_t o0 = (chunk - chunk_pre[blk]) * kMergeChunk, o1 = min(o0 + kMergeChunk, cnt);
    const uint32_t L = (uint32_t)kBlockSortCap << (q - 1);  // run length of this pass
    const uint32_t pa = (uint32_t)(((uint64_t)o0 / (2ull * L)) * 2ull * L);  // start of the run pair
    const uint32_t na = min(L, cnt - pa), nb = cnt - pa > L ? min(L, cnt - pa - L) : 0u;
    const uint32_t d0 = o0 - pa, d1 = o1 - pa;
    const uint64_t hi = ks[0] & 0xFFFFFFFF00000000ull;
    if (nb == 0) {  // a lone run: copy
        for (uint32_t x = o0 + threadIdx.x; x < o1; x += kMergeThreads) {
            kd[x] = ks[x];
            if (VALUES) vd[x] = vs[x];
        }
        return;
    }
    const uint64_t* A = ks + pa;
    const uint64_t* B = ks + pa + L;
    if (threadIdx.x < 2) s_split[threadIdx.x] = merge_split(A, na, B, nb, threadIdx.x ? d1 : d0);
    __syncthreads();
    const uint32_t i0 = s_split[0], i1 = s_split[1];
    const uint32_t j0 = d0 - i0, j1 = d1 - i1;
    const uint32_t ca = i1 - i0, cb = j1 - j0, tot = ca + cb;
    for (uint32_t x = threadIdx.x; x < tot; x += kMergeThreads) {
        const bool in_a = x < ca;
        const uint32_t src = in_a ? pa + i0 + x : pa + L + j0 + (x - ca);
        sk[x] = (uint32_t)ks[src];
        if (VALUES) sv[x] = vs[src];
    }
    __syncthreads();
    // each thread merges kMergeItems outputs from its own split of the staged windows
    const uint32_t dd = min((uint32_t)threadIdx.x * kMergeItems, tot);
    uint32_t ia = merge_split(sk, ca, sk + ca, cb, dd), ib = dd - ia;
    for (uint32_t m = 0; m < (uint32_t)kMergeItems && dd + m < tot; m++) {
        const bool take_a = ib >= cb || (ia < ca && sk[ia] <= sk[ca + ib]);
        const uint32_t from = take_a ? ia++ : ca + ib++;
        ok[dd + m] = sk[from];
        if (VALUES) ov[dd + m] = sv[from];
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < tot; x += kMergeThreads) {
        kd[o0 + x] = hi | ok[x];
        if (VALUES) vd[o0 + x] = ov[x];
    }
}

static_assert(block_sort_smem<true>() <= 48 * 1024 && block_sort_smem<false>() <= 48 * 1024,
              "the tile sort runs without a shared-memory opt-in");

template <bool VALUES>
uint32_t enqueue_t(uint32_t nblk, const uint64_t* off, uint64_t tiles, uint64_t chunks, uint32_t passes,
                   uint32_t* tile_pre, uint32_t* chunk_pre, const uint32_t* unsorted, uint64_t* ka, uint32_t* va,
                   uint64_t* kb, uint32_t* vb, uint32_t* maxp, cudaStream_t st, bool plan) {
    uint32_t launches = 0;
    if (plan) {
        k_sort_plan<<<1, 1024, 0, st>>>(nblk, off, tile_pre, chunk_pre);
        launches++;
    }
    if (!tiles) return launches;
    cudaMemsetAsync(maxp, 0, 4, st);
    k_tile_copy<VALUES><<<(unsigned)tiles, kBsThreads, 0, st>>>(nblk, off, tile_pre, unsorted, ka, va, kb, vb);
    k_tile_sort<VALUES><<<(unsigned)tiles, kBsThreads, block_sort_smem<VALUES>(), st>>>(nblk, off, tile_pre, unsorted,
                                                                                      ka, va, kb, vb, maxp);
    launches += 2;
    for (uint32_t q = 1; q <= passes && chunks; q++) {
        k_merge_pass<VALUES><<<(unsigned)chunks, kMergeThreads, 0, st>>>(q, nblk, off, chunk_pre, unsorted, ka, va, kb,
                                                                       vb, maxp);
        launches++;
    }
    return launches;
}

}  // namespace

uint32_t block_sort_enqueue(uint32_t nblk, const uint64_t* off, uint64_t tiles, uint64_t chunks, uint32_t passes,
                            uint32_t* tile_pre, uint32_t* chunk_pre, const uint32_t* unsorted, uint64_t* ka,
                            uint32_t* va, uint64_t* kb, uint32_t* vb, uint32_t* maxp, cudaStream_t st, bool plan) {
    return va ? enqueue_t<true>(nblk, off, tiles, chunks, passes, tile_pre, chunk_pre, unsorted, ka, va, kb, vb, maxp,
                                st, plan)
              : enqueue_t<false>(nblk, off, tiles, chunks, passes, tile_pre, chunk_pre, unsorted, ka, nullptr, kb,
                                 nullptr, maxp, st, plan);
}

}  // namespace rgl
