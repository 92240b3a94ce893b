// K9: the non-zero cells of the dense Q x D count matrix as a CSR matrix, on the device.
//
// query_database collects, row by row and column by column, every cell with a non-zero count into
// all_entries (src/tasks/query/mod.rs:288-298) and builds a CSR from those (row, column)-sorted
// entries (build_csr_from_sorted_entries, src/tasks/query/sweep.rs:4-23).  Here one warp per row
// counts the row's non-zero cells with ballots, an exclusive scan of the row counts gives the row
// pointers, and a second warp-per-row pass writes column indices, counts and overlap base pairs at
// their ballot ranks, so the entries come out in exactly that (row, column) order.
#include <algorithm>

#include "internal.h"

namespace rgl {
namespace {

// indptr[r + 1] = number of non-zero cells of row r (indptr[0] = 0).
__global__ void k_row_nnz(uint32_t rows, uint32_t D, const uint32_t* __restrict__ counts,
                          unsigned long long* __restrict__ indptr) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp == 0 && lane == 0) indptr[0] = 0;
    if (warp >= rows) return;
    const uint32_t* row = counts + warp * D;
    unsigned long long n = 0;
    for (uint32_t c0 = 0; c0 < D; c0 += 32) {
        const uint32_t c = c0 + lane;
        const bool nz = c < D && __ldg(row + c) != 0u;
        n += __popc(__ballot_sync(0xffffffffu, nz));
    }
    if (lane == 0) indptr[warp + 1] = n;
}

// In-place inclusive scan of indptr[1..rows] by one block: each thread sums a contiguous stretch,
// a block scan of the stretch totals gives each stretch its offset, and the stretch is rewritten.
__global__ void __launch_bounds__(1024) k_scan_rows(uint32_t rows, unsigned long long* __restrict__ indptr) {
    __shared__ unsigned long long part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (rows + 1023) / 1024;
    const uint64_t a = 1 + (uint64_t)t * per, b = std::min<uint64_t>(a + per, (uint64_t)rows + 1);
    unsigned long long s = 0;
    for (uint64_t i = a; i < b; i++) s += indptr[i];
    part[t] = s;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan of the totals
        const unsigned long long v = t >= off ? part[t - off] : 0ull;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned long long run = t ? part[t - 1] : 0ull;
    for (uint64_t i = a; i < b; i++) {
        run += indptr[i];
        indptr[i] = run;
    }
}

// Column indices, counts and base pairs of every non-zero cell at position indptr[row] + its rank
// among the row's non-zero cells; positions at or past `capacity` are not written.
__global__ void k_csr_emit(uint32_t rows, uint32_t D, const uint32_t* __restrict__ counts,
                           const unsigned long long* __restrict__ bp, const unsigned long long* __restrict__ indptr,
                           uint64_t capacity, uint32_t* __restrict__ indices, uint32_t* __restrict__ values,
                           unsigned long long* __restrict__ bp_values) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp >= rows) return;
    const uint32_t* row = counts + warp * D;
    unsigned long long at = indptr[warp];
    for (uint32_t c0 = 0; c0 < D; c0 += 32) {
        const uint32_t c = c0 + lane;
        const uint32_t v = c < D ? __ldg(row + c) : 0u;
        const uint32_t mask = __ballot_sync(0xffffffffu, v != 0u);
        if (v) {
            const unsigned long long p = at + __popc(mask & ((1u << lane) - 1u));
            if (p < capacity) {
                indices[p] = c;
                if (values) values[p] = v;
                if (bp_values) bp_values[p] = bp[warp * D + c];
            }
        }
        at += __popc(mask);
    }
}

}  // namespace
}  // namespace rgl

using namespace rgl;

extern "C" int rgl_dense_to_csr_device(rgl_context* ctx, uint32_t num_rows, uint32_t num_sources,
                                       const uint32_t* d_counts, const uint64_t* d_overlap_bp, uint64_t* d_indptr,
                                       uint32_t* d_indices, uint32_t* d_values, uint64_t* d_bp_values,
                                       uint64_t capacity, uint64_t* out_nnz) {
    clear_error();
    if (!ctx || !d_indptr || !out_nnz || (num_rows && num_sources && !d_counts))
        return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    if (d_bp_values && !d_overlap_bp) return fail(RGL_ERR_INVALID_ARGUMENT, "base-pair values need d_overlap_bp");
    if ((uint64_t)num_rows * num_sources >= (1ull << 40))
        return fail(RGL_ERR_INVALID_ARGUMENT, "num_rows x num_sources must be < 2^40");
    cudaStream_t st = context_stream(ctx);
    unsigned long long* indptr = reinterpret_cast<unsigned long long*>(d_indptr);
    if (num_rows == 0) {
        RGL_CUDA(cudaMemsetAsync(d_indptr, 0, 8, st));
        RGL_CUDA(cudaStreamSynchronize(st));
        *out_nnz = 0;
        return RGL_OK;
    }
    const uint64_t threads = (uint64_t)num_rows * 32;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    k_row_nnz<<<blocks, 256, 0, st>>>(num_rows, num_sources, d_counts, indptr);
    k_scan_rows<<<1, 1024, 0, st>>>(num_rows, indptr);
    if (d_indices)
        k_csr_emit<<<blocks, 256, 0, st>>>(num_rows, num_sources, d_counts,
                                           reinterpret_cast<const unsigned long long*>(d_overlap_bp), indptr,
                                           capacity, d_indices, d_values,
                                           reinterpret_cast<unsigned long long*>(d_bp_values));
    RGL_CUDA(cudaGetLastError());
    uint64_t nnz = 0;
    RGL_CUDA(cudaMemcpyAsync(&nnz, d_indptr + num_rows, 8, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    *out_nnz = nnz;
    if (d_indices && nnz > capacity)
        return fail(RGL_ERR_INVALID_ARGUMENT, "CSR capacity " + std::to_string(capacity) + " < " +
                                                  std::to_string(nnz) + " non-zero cells");
    return RGL_OK;
}
