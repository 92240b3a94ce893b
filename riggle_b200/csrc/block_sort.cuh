// Block-local sort of 64-bit keys (and optional 32-bit values), shared by the query pipeline and the
// batched stats stage.  Every block of the input holds keys with one common high word (the block's
// segment); each block is sorted by the low word, stably, independently of the others.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace rgl {

// For runs in which every input block holds one segment ((shard, row)) and no two blocks share one,
// the segment-major order of a device-wide sort is the blocks' own order with each block sorted by
// position, so the keys are sorted block by block, at any block size:
//   * k_expand_keys marks a block whose starts (ends) are not in order (the usual sorted BED input
//     has its starts in order; its ends are in order unless an interval contains the next one);
//   * k_sort_plan lays the blocks out as tiles of kBlockSortCap intervals and, for blocks of more
//     than one tile, merge chunks of kMergeChunk output positions;
//   * k_tile_sort copies a tile of an ordered block to its place, or sorts it in shared memory (a
//     radix sort over the bits its positions use; a tile already in order is copied through);
//   * merge passes q = 1, 2, ... combine sorted runs of kBlockSortCap << (q - 1) pairwise until each
//     block is one run: every CTA takes kMergeChunk outputs of one run pair, finds where they start
//     in both runs by a merge-path search, and merges them in shared memory.
// Every step is stable (equal positions keep their input order), like the radix sort it replaces.
// A block that needs p merge passes has its tiles written where p ping-pong passes end in the
// output buffer (in place into the input buffer when p is odd), so blocks of different sizes share
// the passes and all finish in the output.
constexpr int kBsThreads = 256, kBsItems = 16;
constexpr uint64_t kBlockSortCap = (uint64_t)kBsThreads * kBsItems;
constexpr int kMergeThreads = 256, kMergeItems = 8;
constexpr uint32_t kMergeChunk = (uint32_t)(kMergeThreads * kMergeItems);
static_assert(kBlockSortCap % kMergeChunk == 0, "a merge chunk lies inside one run pair");

__host__ __device__ inline uint32_t sort_tiles(uint64_t cnt) {
    return (uint32_t)((cnt + kBlockSortCap - 1) / kBlockSortCap);
}
__host__ __device__ inline uint32_t sort_passes(uint64_t cnt) {
    const uint32_t t = sort_tiles(cnt);
    uint32_t p = 0;
    while ((1u << p) < t) p++;
    return p;
}
__host__ __device__ inline uint32_t merge_chunks(uint64_t cnt) {
    return cnt > kBlockSortCap ? (uint32_t)((cnt + kMergeChunk - 1) / kMergeChunk) : 0u;
}

// Enqueues the block sort on `st`: the plan (tile and merge-chunk prefix counts, when `plan`), the
// tiles, then `passes` merge passes.  off: nblk + 1 block offsets; unsorted[b] != 0 marks block b
// as not in order; tiles / chunks / passes: the host's counts for these blocks (sort_tiles,
// merge_chunks, sort_passes of the largest block).  (ka, va) is the input and scratch, (kb, vb) the
// output; va and vb null: keys alone.  maxp: one device word of scratch (the most merge passes an
// out-of-order block needs; passes beyond it return at once), its own for each concurrent sort.
// Returns the number of kernels launched.
uint32_t block_sort_enqueue(uint32_t nblk, const uint64_t* off, uint64_t tiles, uint64_t chunks, uint32_t passes,
                            uint32_t* tile_pre, uint32_t* chunk_pre, const uint32_t* unsorted, uint64_t* ka,
                            uint32_t* va, uint64_t* kb, uint32_t* vb, uint32_t* maxp, cudaStream_t st, bool plan);

}  // namespace rgl
