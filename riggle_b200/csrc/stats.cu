// Analytic p-values (K8): compute_analytic_pvalues (src/tasks/query/pvalues.rs:22-77) and
// compute_analytic_stats (src/fourier/stats.rs:34-126) in FP64 on the device, plus the host pieces
// they need: the compact moment-store layout (src/fourier/moments.rs:58-66, 215-247) and the
// per-chromosome query length groups (build_query_chrom_data, src/fourier/moments.rs:138-177).
//
// Moment store in HBM: one float2 (mean, var) table per (source, chromosome), laid out
// [source][chromosome][slot]; slot = compact_index(L) and the tables hold the reference's L grid in
// store order, so a lookup is one gather.  Query groups are flattened per query row: every group
// carries its chromosome, its slot (computed on the host with the same f64 ln as the reference,
// never on the device) and its FP64 sums.  One warp evaluates one (query row, source) pair:
// lanes stride over the row's groups, accumulate mu, sigma^2 and mu_raw in FP64, reduce, and lane
// 0 dispatches NB / Poisson, evaluates the LLR and the A&S 7.1.26 tail exactly as the reference
// writes it (src/fourier/stats.rs:65-126).
#include <cub/cub.cuh>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "block_sort.cuh"
#include "internal.h"

namespace rgl {

static const uint64_t T_THRESHOLD = 100;  // src/fourier/moments.rs:50
static const double EPS = 0.01;           // src/fourier/moments.rs:47

uint64_t compact_index(uint64_t l) {
    // src/fourier/moments.rs:58-66
    if (l <= T_THRESHOLD) return l - 1;
    uint64_t k = (uint64_t)(std::log((double)l / (double)T_THRESHOLD) / std::log(1.0 + EPS));
    return T_THRESHOLD + k - 1;
}

std::vector<uint64_t> moment_grid(uint64_t n) {
    // src/fourier/moments.rs:215-247: L = 1..=min(T, N-1), then ceil of repeated *1.01 products,
    // deduplicated, while L <= N-1.
    std::vector<uint64_t> ls;
    if (n <= 1) return ls;
    const uint64_t max_l = n - 1;
    for (uint64_t l = 1; l <= std::min(T_THRESHOLD, max_l); l++) ls.push_back(l);
    double l_f = (double)T_THRESHOLD;
    uint64_t prev = T_THRESHOLD;
    for (;;) {
        l_f *= 1.0 + EPS;
        const uint64_t l = (uint64_t)std::ceil(l_f);
        if (l > max_l) break;
        if (l > prev) {
            ls.push_back(l);
            prev = l;
        }
    }
    return ls;
}

struct QGroupDev {
    uint32_t chrom, slot;
    double ss, ss2, l_int, count;
};

__device__ __forceinline__ double erfc_as(double x) {
    // A&S 7.1.26 as src/fourier/stats.rs:116-126 writes it (x >= 0 here)
    const double t = 1.0 / (1.0 + 0.3275911 * x);
    const double p =
        t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
    return p * exp(-x * x);
}

__device__ __forceinline__ double ln_half_erfc_as(double x) {
    // ln(erfc_as(x) / 2) without underflow: ln(0.5 t poly(t)) - x*x
    const double t = 1.0 / (1.0 + 0.3275911 * x);
    const double p =
        t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
    return log(0.5 * p) + (-x * x);
}

__global__ void k_pvalues(uint32_t rows, uint32_t D, uint32_t C, const uint32_t* __restrict__ counts,
                          const unsigned long long* __restrict__ bp, double bin_size,
                          const uint64_t* __restrict__ g_off, const QGroupDev* __restrict__ groups,
                          const float2* __restrict__ mv, const uint64_t* __restrict__ chrom_off, uint64_t stride,
                          const uint32_t* __restrict__ tab_len, double* __restrict__ p_out,
                          double* __restrict__ llr_out, double* __restrict__ logp_out, uint8_t* __restrict__ flags) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; w < (uint64_t)rows * D; w += nw) {
        const uint32_t q = (uint32_t)(w / D), d = (uint32_t)(w % D);
        const uint32_t cnt = counts[w];
        double p = 1.0, llr = 0.0, lp = 0.0;
        uint8_t f = 0;
        if (cnt) {  // zero-count pairs are not emitted (src/tasks/query/pvalues.rs:28-35)
            double mu = 0.0, var = 0.0, raw = 0.0;
            uint32_t any = 0;
            const float2* src = mv + (uint64_t)d * stride;
            for (uint64_t g = g_off[q] + lane; g < g_off[q + 1]; g += 32) {
                const QGroupDev G = groups[g];
                if (G.slot < tab_len[(uint64_t)d * C + G.chrom]) {
                    const float2 m = src[chrom_off[G.chrom] + G.slot];
                    const double mean = (double)m.x, v = (double)m.y;
                    mu += mean * G.ss;
                    var += v * G.ss2;
                    raw += mean / G.l_int * G.count;
                    any = 1;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                mu += __shfl_xor_sync(0xffffffffu, mu, o);
                var += __shfl_xor_sync(0xffffffffu, var, o);
                raw += __shfl_xor_sync(0xffffffffu, raw, o);
                any |= __shfl_xor_sync(0xffffffffu, any, o);
            }
            if (any) {
                f = 1;
                const double observed = (double)bp[w] / bin_size;
                bool ok = false;
                if (var > mu) {
                    // nb_llr (src/fourier/stats.rs:101-113)
                    if (mu > 0.0 && var > mu) {
                        const double r = mu * mu / (var - mu);
                        const double pp = mu / var;
                        const double p_o = r / (r + observed);
                        if (0.0 < pp && pp < 1.0 && 0.0 < p_o && p_o < 1.0) {
                            const double theta = log((1.0 - p_o) / (1.0 - pp));
                            llr = observed * theta + r * log(p_o / pp);
                            ok = true;
                        }
                    }
                } else {
                    // Poisson on count units (src/fourier/stats.rs:65-74, 93-98)
                    const double eff = raw > 0.0 ? mu / raw : 1.0;
                    const double oc = observed / eff;
                    if (raw > 0.0 && oc > 0.0) {
                        llr = oc * log(oc / raw) - (oc - raw);
                        ok = true;
                    }
                }
                if (ok) f |= 2;
                if (ok && llr > 0.0) {
                    const double x = sqrt(llr);
                    const double tail = erfc_as(x) * 0.5;
                    const double ln_tail = ln_half_erfc_as(x);
                    if (observed >= mu) {
                        p = tail;
                        lp = ln_tail;
                    } else {
                        p = 1.0 - tail;
                        lp = log1p(-exp(ln_tail));
                    }
                }
                if (!ok) llr = 0.0;
            }
        }
        if (lane == 0) {
            p_out[w] = p;
            llr_out[w] = llr;
            if (logp_out) logp_out[w] = lp;
            flags[w] = f;
        }
    }
}

// ---- query length groups of a whole device-resident batch ------------------------------------
// build_query_chrom_data (src/fourier/moments.rs:138-177) groups a file's lengths on one chromosome
// by l_int = max(ceil(len / bin), 1) and sums s = (len / bin) / l_int and s^2.  Here every interval
// of the batch gets the key (row * C + chrom) << 32 | l_int, the keys are sorted and each run is
// reduced with exact integer sums of len and len^2, so that sum_s = sum_len / (bin * l_int) and
// sum_s2 = sum_len2 / (bin * l_int)^2 carry one rounding each instead of the reference's sequential
// f64 rounding (they agree to ~1e-15 relative).
struct LenAgg {
    unsigned long long cnt, s1, s2lo, s2hi;  // count, sum of len, sum of len^2 (128-bit)
};
struct LenAggOp {
    __device__ __forceinline__ LenAgg operator()(const LenAgg& a, const LenAgg& b) const {
        LenAgg r;
        r.cnt = a.cnt + b.cnt;
        r.s1 = a.s1 + b.s1;
        r.s2lo = a.s2lo + b.s2lo;
        r.s2hi = a.s2hi + b.s2hi + (r.s2lo < a.s2lo ? 1ull : 0ull);
        return r;
    }
};
struct LenToAgg {
    __host__ __device__ __forceinline__ LenAgg operator()(uint32_t len) const {
        const unsigned long long l = len;
        return LenAgg{1ull, l, l * l, 0ull};  // len < 2^32: len^2 fits 64 bits
    }
};

constexpr uint64_t kNoGroup = ~0ull;
constexpr uint32_t kNoLen = 0xFFFFFFFFu;  // block-local keys: the low word of an interval in no group
// the request server sizes each worker's StatsScratch with these record sizes
static_assert(sizeof(LenAgg) == 32 && sizeof(QGroupDev) == 40, "stats scratch record sizes changed");

__global__ void k_group_keys(uint64_t n, const rgl_interval* __restrict__ iv, const uint64_t* __restrict__ blk_off,
                             const uint32_t* __restrict__ blk_shard, const uint32_t* __restrict__ blk_row, uint32_t nblk,
                             const uint32_t* __restrict__ shard_chrom, uint32_t nshards, uint32_t C,
                             const uint64_t* __restrict__ n_bins, double bin, int local, uint64_t* __restrict__ key,
                             uint32_t* __restrict__ len_out) {
    // last block with blk_off[b] <= j: one search per thread block, for its first element, then a
    // short walk (256 consecutive intervals span few blocks)
    __shared__ uint32_t s_b0;
    const uint64_t j0 = blockIdx.x * (uint64_t)blockDim.x, j = j0 + threadIdx.x;
    if (threadIdx.x == 0) {
        uint32_t lo = 0, hi = nblk;
        while (hi - lo > 1) {
            const uint32_t m = (lo + hi) >> 1;
            if (blk_off[m] <= j0) lo = m; else hi = m;
        }
        s_b0 = lo;
    }
    __syncthreads();
    if (j >= n) return;
    uint32_t lo = s_b0;
    while (lo + 1 < nblk && blk_off[lo + 1] <= j) lo++;
    const rgl_interval v = iv[j];
    const uint32_t sh = blk_shard[lo];
    const uint32_t c = sh < nshards ? shard_chrom[sh] : 0xFFFFFFFFu;
    uint64_t k = kNoGroup;
    const uint32_t len = v.end > v.start ? v.end - v.start : 0u;
    if (c < C && len) {
        const double l = (double)len / bin;  // as build_query_chrom_data: lengths in bins, f64
        const double ce = ceil(l);
        const uint64_t li = ce < 1.0 ? 1ull : (uint64_t)ce;
        // groups with l_int >= n_bins never meet a moment (src/io/momentstore.rs:66-79)
        if (li < n_bins[c]) k = (((uint64_t)blk_row[lo] * C + c) << 32) | li;
    }
    // block-local form: every key of a block carries the block's (row, chromosome) in its high word
    // (all ones without a chromosome), an interval that joins no group kNoLen in its low word
    if (local && k == kNoGroup)
        k = ((c < C ? (uint64_t)blk_row[lo] * C + c : 0xFFFFFFFFull) << 32) | kNoLen;
    key[j] = k;
    len_out[j] = len;
}

// ---- the groups of block-sorted keys ------------------------------------------------------------
// After the block-local sort every block's keys are in ascending l_int order, and the blocks come in
// ascending (row, chromosome) order: the groups are the runs of equal keys, in order.  Run heads
// are counted per tile of the sort (k_run_count), the counts scanned (k_scan_small), heads and tails
// placed (k_run_emit) and each run summed by one warp (k_run_agg), with the exact integer sums of
// the device-wide form.
constexpr int kRunThreads = 256;

__device__ inline uint32_t tile_block(const uint32_t* __restrict__ pre, uint32_t nblk, uint32_t x) {
    uint32_t lo = 0, hi = nblk;  // pre[lo] <= x < pre[lo + 1]
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (__ldg(pre + m) <= x) lo = m; else hi = m;
    }
    return lo;
}

// Whether sorted element g (block [bbeg, bend)) starts a run / ends a run of a usable key.
__device__ inline bool run_head(const uint64_t* __restrict__ key, uint64_t bbeg, uint64_t g) {
    const uint64_t k = key[g];
    return (uint32_t)k != kNoLen && (g == bbeg || key[g - 1] != k);
}
__device__ inline bool run_tail(const uint64_t* __restrict__ key, uint64_t bend, uint64_t g) {
    const uint64_t k = key[g];
    return (uint32_t)k != kNoLen && (g + 1 == bend || key[g + 1] != k);
}

// tile_heads[t] = run heads among the elements of tile t (tiles of kBlockSortCap per block).
__global__ void __launch_bounds__(kRunThreads) k_run_count(uint32_t nblk, const uint64_t* __restrict__ blk_off,
                                                           const uint32_t* __restrict__ tile_pre,
                                                           const uint64_t* __restrict__ key,
                                                           uint32_t* __restrict__ tile_heads) {
    const uint32_t t = blockIdx.x;
    if (t >= __ldg(tile_pre + nblk)) return;
    const uint32_t b = tile_block(tile_pre, nblk, t);
    const uint64_t bbeg = blk_off[b], bend = blk_off[b + 1];
    const uint64_t base = bbeg + (uint64_t)(t - tile_pre[b]) * kBlockSortCap;
    const uint32_t cnt = (uint32_t)min((uint64_t)kBlockSortCap, bend - base);
    uint32_t total = 0;
    for (uint32_t i0 = 0; i0 < cnt; i0 += kRunThreads) {
        const uint32_t i = i0 + threadIdx.x;
        total += __syncthreads_count(i < cnt && run_head(key, bbeg, base + i));
    }
    if (threadIdx.x == 0) tile_heads[t] = total;
}

// out[0..n] = exclusive prefix sums of in[0..n) (out[n] = the total), by one thread block.
__global__ void __launch_bounds__(1024) k_scan_small(uint32_t n, const uint32_t* __restrict__ in,
                                                     uint32_t* __restrict__ out) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (n + 1023) / 1024;
    const uint32_t a = min(t * per, n), b = min(a + per, n);
    uint32_t s = 0;
    for (uint32_t i = a; i < b; i++) s += in[i];
    part[t] = s;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan of the totals
        const uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = t ? part[t - 1] : 0u;
    for (uint32_t i = a; i < b; i++) {
        out[i] = run;
        run += in[i];
    }
    if (t == 1023) out[n] = part[1023];
}

// Run g: ukey[g] its key, bounds[2 g], bounds[2 g + 1] its first and one-past-last element.
__global__ void __launch_bounds__(kRunThreads) k_run_emit(uint32_t nblk, const uint64_t* __restrict__ blk_off,
                                                          const uint32_t* __restrict__ tile_pre,
                                                          const uint32_t* __restrict__ tile_off,
                                                          const uint64_t* __restrict__ key,
                                                          uint64_t* __restrict__ ukey, uint32_t* __restrict__ bounds) {
    using Scan = cub::BlockScan<uint32_t, kRunThreads>;
    __shared__ typename Scan::TempStorage tmp;
    const uint32_t t = blockIdx.x;
    if (t >= __ldg(tile_pre + nblk)) return;
    const uint32_t b = tile_block(tile_pre, nblk, t);
    const uint64_t bbeg = blk_off[b], bend = blk_off[b + 1];
    const uint64_t base = bbeg + (uint64_t)(t - tile_pre[b]) * kBlockSortCap;
    const uint32_t cnt = (uint32_t)min((uint64_t)kBlockSortCap, bend - base);
    uint32_t at = tile_off[t];  // runs started before this 256-element step
    for (uint32_t i0 = 0; i0 < cnt; i0 += kRunThreads) {
        const uint32_t i = i0 + threadIdx.x;
        const uint64_t g = base + i;
        const bool head = i < cnt && run_head(key, bbeg, g);
        const bool tail = i < cnt && run_tail(key, bend, g);
        uint32_t excl, step;
        Scan(tmp).ExclusiveSum(head ? 1u : 0u, excl, step);
        if (head) {
            ukey[at + excl] = key[g];
            bounds[2ull * (at + excl)] = (uint32_t)g;
        }
        // the run a tail closes: the last head at or before it
        if (tail) bounds[2ull * (at + excl + (head ? 1u : 0u) - 1u) + 1] = (uint32_t)(g + 1);
        at += step;
        __syncthreads();  // tmp is reused by the next step's scan
    }
}

// One warp per run (grid-stride): count, sum of lengths and 128-bit sum of squared lengths.
__global__ void __launch_bounds__(kRunThreads) k_run_agg(const uint32_t* __restrict__ num_runs,
                                                         const uint32_t* __restrict__ bounds,
                                                         const uint32_t* __restrict__ len, LenAgg* __restrict__ agg) {
    const uint32_t runs = *num_runs;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < runs; g += warps) {
        const uint32_t a = bounds[2 * g], e = bounds[2 * g + 1];
        unsigned long long c = 0, s1 = 0, lo = 0, hi = 0;
        for (uint32_t j = a + lane; j < e; j += 32) {
            const unsigned long long l = len[j], q = l * l;
            c++;
            s1 += l;
            lo += q;
            hi += lo < q ? 1ull : 0ull;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            c += __shfl_down_sync(0xffffffffu, c, o);
            s1 += __shfl_down_sync(0xffffffffu, s1, o);
            const unsigned long long plo = __shfl_down_sync(0xffffffffu, lo, o);
            const unsigned long long phi = __shfl_down_sync(0xffffffffu, hi, o);
            lo += plo;
            hi += phi + (lo < plo ? 1ull : 0ull);
        }
        if (lane == 0) agg[g] = LenAgg{c, s1, lo, hi};
    }
}

// One thread per group: FP64 sums, the host-made slot table, and the per-row group offsets.
__global__ void k_group_finish(const uint64_t* __restrict__ ukey, const LenAgg* __restrict__ agg,
                               const uint32_t* __restrict__ num_runs, uint32_t rows, uint32_t C, double bin,
                               const uint32_t* __restrict__ slot_tab, uint64_t slot_tab_len,
                               QGroupDev* __restrict__ groups, uint64_t* __restrict__ g_off) {
    const uint32_t runs = *num_runs;
    // a trailing run of unusable intervals (key kNoGroup) sorts last and is dropped
    const uint32_t ng = (runs && ukey[runs - 1] == kNoGroup) ? runs - 1 : runs;
    const uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (g > ng) return;
    if (g == ng) {  // rows after the last group's row
        const uint32_t r0 = ng ? (uint32_t)((ukey[ng - 1] >> 32) / C) + 1 : 0;
        for (uint32_t r = r0; r <= rows; r++) g_off[r] = ng;
        return;
    }
    const uint64_t k = ukey[g];
    const uint32_t rc = (uint32_t)(k >> 32), row = rc / C, chrom = rc % C;
    const uint64_t li = k & 0xFFFFFFFFull;
    const LenAgg a = agg[g];
    const double den = bin * (double)li;
    const double s2 = (double)a.s2hi * 18446744073709551616.0 + (double)a.s2lo;
    groups[g] = QGroupDev{chrom, li < slot_tab_len ? slot_tab[li] : 0xFFFFFFFFu, (double)a.s1 / den,
                          s2 / (den * den), (double)li, (double)a.cnt};
    const uint32_t prev = g ? (uint32_t)((ukey[g - 1] >> 32) / C) : 0xFFFFFFFFu;
    if (prev != row)  // rows (prev, row] start at this group
        for (uint32_t r = (prev == 0xFFFFFFFFu ? 0 : prev + 1); r <= row; r++) g_off[r] = g;
}

}  // namespace rgl

using namespace rgl;

struct rgl_moments {
    int device = 0;
    uint32_t num_sources = 0, num_chroms = 0;
    std::vector<uint64_t> n_bins, n_slots, chrom_off;
    uint64_t stride = 0;
    float2* d_mv = nullptr;
    uint32_t* d_len = nullptr;
    std::vector<uint32_t> len;  // host mirror of the per-(source, chromosome) table lengths
    // batched stats: compact_index table (slot of every l_int below the largest n_bins), chromosome
    // offsets and bin counts on the device (built once, under tab_mu), and the scratch of the
    // public entry points (a request server gives each worker its own)
    DevBuf slot_tab, coff, nb;
    uint64_t lmax = 1;
    bool tables_ready = false;
    std::mutex tab_mu;
    StatsScratch sc;
};

namespace rgl {
// Device pointer of the (sid, chrom) table of a moment store and its full grid length.
int moments_table_ptr(rgl_moments* m, uint32_t sid, uint32_t chrom, float2** ptr, uint64_t* slots, uint64_t* n_bins,
                      int* device) {
    if (!m || sid >= m->num_sources || chrom >= m->num_chroms) return fail(RGL_ERR_INVALID_ARGUMENT, "bad moment table");
    *ptr = m->d_mv + (uint64_t)sid * m->stride + m->chrom_off[chrom];
    *slots = m->n_slots[chrom];
    *n_bins = m->n_bins[chrom];
    *device = m->device;
    return RGL_OK;
}
// Records that (sid, chrom) now holds `entries` entries.
int moments_mark(rgl_moments* m, uint32_t sid, uint32_t chrom, uint64_t entries) {
    const uint32_t l = (uint32_t)entries;
    m->len[(size_t)sid * m->num_chroms + chrom] = l;
    RGL_CUDA(cudaMemcpy(m->d_len + (size_t)sid * m->num_chroms + chrom, &l, 4, cudaMemcpyHostToDevice));
    return RGL_OK;
}
}  // namespace rgl

extern "C" {

uint64_t rgl_compact_index(uint64_t l) { return l ? compact_index(l) : 0; }

uint64_t rgl_moment_grid(uint64_t n_bins, uint64_t* out, uint64_t cap) {
    auto g = moment_grid(n_bins);
    for (uint64_t i = 0; i < g.size() && i < cap && out; i++) out[i] = g[i];
    return g.size();
}

int rgl_query_chrom_groups(const rgl_interval* ivs, uint64_t n, uint32_t bin_size, uint64_t* l_int,
                           double* sum_scale, double* sum_scale2, uint64_t* count, uint64_t capacity,
                           uint64_t* out_groups) {
    // build_query_chrom_data inner loop (src/fourier/moments.rs:148-172): lengths in bins sorted
    // ascending, grouped by l_int = max(ceil(l), 1), with sums of s = l / l_int and s^2.
    clear_error();
    if ((!ivs && n) || !out_groups || bin_size == 0) return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    std::vector<double> lengths(n);
    for (uint64_t i = 0; i < n; i++) {
        if (ivs[i].end <= ivs[i].start) return fail(RGL_ERR_INVALID_ARGUMENT, "interval with start >= end");
        lengths[i] = (double)(ivs[i].end - ivs[i].start) / (double)bin_size;
    }
    std::sort(lengths.begin(), lengths.end());
    auto lint_of = [](double l) {
        uint64_t c = (uint64_t)std::ceil(l);
        return c < 1 ? (uint64_t)1 : c;
    };
    uint64_t ng = 0;
    for (uint64_t i = 0; i < n;) {
        const double l = lengths[i];
        const uint64_t li = lint_of(l);
        const double s0 = l / (double)li;
        double ss = s0, ss2 = s0 * s0;
        uint64_t c = 1;
        for (i++; i < n && lint_of(lengths[i]) == li; i++) {
            const double s = lengths[i] / (double)li;
            ss += s;
            ss2 += s * s;
            c++;
        }
        if (ng < capacity) {
            if (l_int) l_int[ng] = li;
            if (sum_scale) sum_scale[ng] = ss;
            if (sum_scale2) sum_scale2[ng] = ss2;
            if (count) count[ng] = c;
        }
        ng++;
    }
    *out_groups = ng;
    if (ng > capacity && (l_int || sum_scale || sum_scale2 || count))
        return fail(RGL_ERR_INVALID_ARGUMENT, "group capacity too small");
    return RGL_OK;
}

int rgl_moments_create(int device, uint32_t num_sources, uint32_t num_chroms, const uint64_t* n_bins,
                       rgl_moments** out) {
    clear_error();
    if (!out || !n_bins || !num_chroms) return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RGL_ERR_NO_DEVICE, "no CUDA device");
    auto* m = new rgl_moments();
    m->device = device;
    m->num_sources = num_sources;
    m->num_chroms = num_chroms;
    uint64_t acc = 0;
    for (uint32_t c = 0; c < num_chroms; c++) {
        m->n_bins.push_back(n_bins[c]);
        const uint64_t ns = moment_grid(n_bins[c]).size();
        m->n_slots.push_back(ns);
        m->chrom_off.push_back(acc);
        acc += ns;
    }
    m->stride = acc;
    m->len.assign((size_t)num_sources * num_chroms, 0);
    int s = RGL_OK;
    if (cudaSetDevice(device) != cudaSuccess) s = fail(RGL_ERR_DEVICE, "cudaSetDevice");
    size_t mv_bytes = std::max<size_t>(1, (size_t)num_sources * acc) * sizeof(float2);
    size_t len_bytes = std::max<size_t>(1, m->len.size()) * 4;
    if (s == RGL_OK && cudaMalloc(&m->d_mv, mv_bytes) != cudaSuccess) s = fail(RGL_ERR_OOM, "moment store");
    if (s == RGL_OK && cudaMalloc(&m->d_len, len_bytes) != cudaSuccess) s = fail(RGL_ERR_OOM, "moment store");
    if (s == RGL_OK && cudaMemset(m->d_len, 0, len_bytes) != cudaSuccess) s = fail(RGL_ERR_DEVICE, "memset");
    if (s != RGL_OK) {
        if (m->d_mv) cudaFree(m->d_mv);
        if (m->d_len) cudaFree(m->d_len);
        delete m;
        return s;
    }
    *out = m;
    return RGL_OK;
}

int rgl_moments_destroy(rgl_moments* m) {
    clear_error();
    if (!m) return RGL_OK;
    cudaSetDevice(m->device);
    for (DevBuf* b : {&m->slot_tab, &m->coff, &m->nb}) b->release();
    stats_scratch_release(&m->sc);
    if (m->d_mv) cudaFree(m->d_mv);
    if (m->d_len) cudaFree(m->d_len);
    delete m;
    return RGL_OK;
}

uint64_t rgl_moments_slots(const rgl_moments* m, uint32_t chrom) {
    return (m && chrom < m->num_chroms) ? m->n_slots[chrom] : 0;
}

int rgl_moments_set(rgl_moments* m, uint32_t sid, uint32_t chrom, const float* mean_var, uint64_t entries) {
    // MomentStoreBuilder::insert for one (source, chromosome) (src/io/momentstore.rs:134-154)
    clear_error();
    if (!m || sid >= m->num_sources || chrom >= m->num_chroms || (entries && !mean_var))
        return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    if (entries > m->n_slots[chrom])
        return fail(RGL_ERR_INVALID_ARGUMENT, "more entries than the chromosome's L grid");
    RGL_CUDA(cudaSetDevice(m->device));
    if (entries)
        RGL_CUDA(cudaMemcpy(m->d_mv + (uint64_t)sid * m->stride + m->chrom_off[chrom], mean_var, entries * 8,
                            cudaMemcpyHostToDevice));
    const uint32_t l = (uint32_t)entries;
    m->len[(size_t)sid * m->num_chroms + chrom] = l;
    RGL_CUDA(cudaMemcpy(m->d_len + (size_t)sid * m->num_chroms + chrom, &l, 4, cudaMemcpyHostToDevice));
    return RGL_OK;
}

int rgl_moments_get(const rgl_moments* m, uint32_t sid, uint32_t chrom, float* mean_var, uint64_t capacity,
                    uint64_t* out_entries) {
    clear_error();
    if (!m || sid >= m->num_sources || chrom >= m->num_chroms || !out_entries)
        return fail(RGL_ERR_INVALID_ARGUMENT, "bad arguments");
    const uint64_t l = m->len[(size_t)sid * m->num_chroms + chrom];
    *out_entries = l;
    if (!mean_var || !l) return RGL_OK;
    if (capacity < l) return fail(RGL_ERR_INVALID_ARGUMENT, "capacity too small");
    RGL_CUDA(cudaSetDevice(m->device));
    RGL_CUDA(cudaMemcpy(mean_var, m->d_mv + (uint64_t)sid * m->stride + m->chrom_off[chrom], l * 8,
                        cudaMemcpyDeviceToHost));
    return RGL_OK;
}

int rgl_query_pvalues(rgl_moments* m, const rgl_pvalue_batch* b, uint32_t bin_size, const uint32_t* counts,
                      const uint64_t* overlap_bp, double* p, double* llr, double* log_p, uint8_t* flags) {
    clear_error();
    if (!m || !b || !counts || !overlap_bp || !p || !llr || !flags || bin_size == 0)
        return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    const uint32_t rows = b->num_rows, D = m->num_sources, C = m->num_chroms;
    const uint64_t cells = (uint64_t)rows * D;
    if (!cells) return RGL_OK;
    // flatten the groups: validity on the host (l_int < n_bins of the chromosome, as the store's
    // lookup requires, src/io/momentstore.rs:66-79); slot by compact_index
    std::vector<uint64_t> goff(rows + 1, 0);
    std::vector<QGroupDev> gs;
    for (uint32_t q = 0; q < rows; q++) {
        goff[q] = gs.size();
        for (uint64_t g = b->row_group_offsets[q]; g < b->row_group_offsets[q + 1]; g++) {
            const uint32_t c = b->group_chrom[g];
            if (c >= C) return fail(RGL_ERR_INVALID_ARGUMENT, "group chromosome out of range");
            const uint64_t l = b->group_l_int[g];
            if (l == 0 || l >= m->n_bins[c]) continue;
            const uint64_t slot = compact_index(l);
            if (slot >= m->n_slots[c]) continue;
            gs.push_back(QGroupDev{c, (uint32_t)slot, b->group_sum_scale[g], b->group_sum_scale2[g], (double)l,
                                   (double)b->group_count[g]});
        }
    }
    goff[rows] = gs.size();
    RGL_CUDA(cudaSetDevice(m->device));
    DevBuf d_goff, d_g, d_coff, d_cnt, d_bp, d_p, d_llr, d_lp, d_f;
    int s = RGL_OK;
    if (s == RGL_OK) s = d_goff.ensure((rows + 1) * 8ull);
    if (s == RGL_OK) s = d_g.ensure(std::max<size_t>(1, gs.size()) * sizeof(QGroupDev));
    if (s == RGL_OK) s = d_coff.ensure(C * 8ull);
    if (s == RGL_OK) s = d_cnt.ensure(cells * 4);
    if (s == RGL_OK) s = d_bp.ensure(cells * 8);
    if (s == RGL_OK) s = d_p.ensure(cells * 8);
    if (s == RGL_OK) s = d_llr.ensure(cells * 8);
    if (s == RGL_OK) s = d_lp.ensure(cells * 8);
    if (s == RGL_OK) s = d_f.ensure(cells);
    auto cp = [&](void* dst, const void* src, size_t n) {
        if (s == RGL_OK && n && cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice) != cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "p-value upload");
    };
    cp(d_goff.p, goff.data(), goff.size() * 8);
    cp(d_g.p, gs.data(), gs.size() * sizeof(QGroupDev));
    cp(d_coff.p, m->chrom_off.data(), C * 8);
    cp(d_cnt.p, counts, cells * 4);
    cp(d_bp.p, overlap_bp, cells * 8);
    if (s == RGL_OK) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
        const uint64_t warps = std::min<uint64_t>(cells, (uint64_t)nsm * 64);
        k_pvalues<<<(unsigned)((warps * 32 + 255) / 256), 256>>>(
            rows, D, C, d_cnt.as<uint32_t>(), d_bp.as<unsigned long long>(), (double)bin_size, d_goff.as<uint64_t>(),
            d_g.as<QGroupDev>(), m->d_mv, d_coff.as<uint64_t>(), m->stride, m->d_len, d_p.as<double>(),
            d_llr.as<double>(), d_lp.as<double>(), d_f.as<uint8_t>());
        if (cudaGetLastError() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "k_pvalues launch");
    }
    auto back = [&](void* dst, const void* src, size_t n) {
        if (s == RGL_OK && dst && cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost) != cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "p-value download");
    };
    back(p, d_p.p, cells * 8);
    back(llr, d_llr.p, cells * 8);
    back(log_p, d_lp.p, cells * 8);
    back(flags, d_f.p, cells);
    for (DevBuf* x : {&d_goff, &d_g, &d_coff, &d_cnt, &d_bp, &d_p, &d_llr, &d_lp, &d_f}) x->release();
    return s;
}

}  // extern "C"

namespace rgl {

void stats_scratch_release(StatsScratch* sc) {
    for (DevBuf* b : {&sc->key_a, &sc->key_b, &sc->len_a, &sc->len_b, &sc->ukey, &sc->agg, &sc->runs, &sc->groups,
                      &sc->goff, &sc->tmp, &sc->plan})
        b->release();
}

// The device tables the batched stats stage reads: compact_index(l) for every l below the largest
// chromosome's n_bins (on the host with the reference's f64 ln), chromosome offsets and bin counts.
// Built once; later calls (any thread) return at once.
int moments_prepare(rgl_moments* m) {
    std::lock_guard<std::mutex> lk(m->tab_mu);
    if (m->tables_ready) return RGL_OK;
    DeviceScope scope;
    RGL_TRY(scope.enter(m->device));
    const uint32_t C = m->num_chroms;
    uint64_t lmax = 1;
    for (uint32_t c = 0; c < C; c++) lmax = std::max(lmax, m->n_bins[c]);
    std::vector<uint32_t> tab(lmax);
    tab[0] = 0xFFFFFFFFu;
    for (uint64_t l = 1; l < lmax; l++) tab[l] = (uint32_t)compact_index(l);
    RGL_TRY(m->slot_tab.ensure(lmax * 4));
    RGL_CUDA(cudaMemcpy(m->slot_tab.p, tab.data(), lmax * 4, cudaMemcpyHostToDevice));
    RGL_TRY(m->coff.ensure(C * 8ull + 8));
    RGL_CUDA(cudaMemcpy(m->coff.p, m->chrom_off.data(), C * 8ull, cudaMemcpyHostToDevice));
    RGL_TRY(m->nb.ensure(C * 8ull + 8));
    RGL_CUDA(cudaMemcpy(m->nb.p, m->n_bins.data(), C * 8ull, cudaMemcpyHostToDevice));
    m->lmax = lmax;
    m->tables_ready = true;
    return RGL_OK;
}

}  // namespace rgl

// Enqueues the query length groups of a device batch on the context stream: m->groups holds them
// (row-major, ascending (chromosome, l_int) within a row) and d_goff[0..rows] the per-row group
// offsets.  *empty is set when there is nothing to do (no rows or no sources).
static int enqueue_batch_groups(rgl_context* ctx, rgl_moments* m, StatsScratch* sc, const rgl_batch* b,
                                const uint32_t* shard_chrom, uint32_t num_shards, uint32_t bin_size, bool* empty,
                                uint64_t** goff_out) {
    if (!ctx || !m || !b || !bin_size || (num_shards && !shard_chrom))
        return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *empty = false;
    if (b->num_blocks && (!b->block_offsets || !b->block_shards || !b->d_intervals))
        return fail(RGL_ERR_INVALID_ARGUMENT, "incomplete batch");
    const uint32_t rows = b->num_rows, D = m->num_sources, C = m->num_chroms;
    const uint64_t n = b->num_blocks ? b->block_offsets[b->num_blocks] - b->block_offsets[0] : 0;
    if ((uint64_t)rows * C >= (1ull << 32)) return fail(RGL_ERR_INVALID_ARGUMENT, "num_rows x chromosomes must be < 2^32");
    if (n >= (1ull << 31)) return fail(RGL_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 intervals per call");
    for (uint32_t i = 0; i < b->num_blocks; i++) {
        if (b->block_offsets[i + 1] < b->block_offsets[i])
            return fail(RGL_ERR_INVALID_ARGUMENT, "block offsets must be non-decreasing");
        if (b->block_rows && b->block_rows[i] >= rows) return fail(RGL_ERR_INVALID_ARGUMENT, "block row >= num_rows");
    }
    if (!b->block_rows && b->num_blocks) return fail(RGL_ERR_INVALID_ARGUMENT, "batched p-values need block_rows");
    if (!rows || !D) {
        *empty = true;
        return RGL_OK;
    }
    RGL_CUDA(cudaSetDevice(m->device));
    cudaStream_t st = context_stream(ctx);
    // slot table: compact_index(l) on the host with the reference's f64 ln, for every l below the
    // largest chromosome's n_bins; slots past a chromosome's grid are rejected per group below
    RGL_TRY(moments_prepare(m));
    const uint64_t lmax = m->lmax;
    const uint32_t nblk = b->num_blocks;
    std::vector<uint64_t> off(nblk + 1);
    for (uint32_t i = 0; i <= nblk; i++) off[i] = b->block_offsets[i] - b->block_offsets[0];
    std::vector<uint32_t> tabs(2ull * nblk + num_shards + 1, 0);
    for (uint32_t i = 0; i < nblk; i++) {
        tabs[i] = b->block_shards[i];
        tabs[nblk + i] = b->block_rows[i];
    }
    for (uint32_t i = 0; i < num_shards; i++) tabs[2ull * nblk + i] = shard_chrom[i];
    // block-local form: every non-empty block with a chromosome holds one (row, chromosome), in
    // ascending order, so sorting within the blocks orders the whole batch
    bool local = true;
    uint64_t tiles = 0, chunks = 0, max_block = 0, prev = 0;
    bool any = false;
    for (uint32_t i = 0; i < nblk && local; i++) {
        const uint64_t cnt = off[i + 1] - off[i];
        tiles += sort_tiles(cnt);
        chunks += merge_chunks(cnt);
        max_block = std::max(max_block, cnt);
        const uint32_t sh = b->block_shards[i];
        const uint32_t c = sh < num_shards ? shard_chrom[sh] : 0xFFFFFFFFu;
        if (!cnt || c >= C) continue;
        const uint64_t rc = (uint64_t)b->block_rows[i] * C + c;
        if (any && rc <= prev) local = false;
        prev = rc;
        any = true;
    }
    if ((uint64_t)rows * C >= 0xFFFFFFFFull) local = false;  // all ones marks blocks without a chromosome
    const uint64_t nn = std::max<uint64_t>(n, 1);
    RGL_TRY(sc->key_a.ensure(nn * 8));
    RGL_TRY(sc->key_b.ensure(nn * 8));
    RGL_TRY(sc->len_a.ensure(nn * 4));
    RGL_TRY(sc->len_b.ensure(nn * 4));
    RGL_TRY(sc->ukey.ensure(nn * 8));
    RGL_TRY(sc->agg.ensure(nn * sizeof(LenAgg)));
    RGL_TRY(sc->groups.ensure(nn * sizeof(QGroupDev)));
    RGL_TRY(sc->goff.ensure((rows + 1ull) * 8 + (nblk + 1ull) * 8 + tabs.size() * 4 + 64));
    RGL_TRY(sc->runs.ensure(64));
    if (local) RGL_TRY(sc->plan.ensure((3ull * nblk + 2 * tiles + 8) * 4));
    uint64_t* d_goff = sc->goff.as<uint64_t>();
    uint64_t* d_boff = d_goff + rows + 1;
    uint32_t* d_tabs = reinterpret_cast<uint32_t*>(d_boff + nblk + 1);
    RGL_CUDA(cudaMemcpyAsync(d_boff, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st));
    RGL_CUDA(cudaMemcpyAsync(d_tabs, tabs.data(), tabs.size() * 4, cudaMemcpyHostToDevice, st));
    thrust::transform_iterator<LenToAgg, const uint32_t*, LenAgg> vin(sc->len_b.as<uint32_t>(), LenToAgg());
    int segbits = 1;
    if (!local) {
        // 2^segbits > rows * C: every valid key's high part is below all ones, so kNoGroup (all bits
        // set) sorts strictly after every valid key within the sorted 32 + segbits bits
        while (segbits < 32 && (1ull << segbits) <= (uint64_t)rows * C) segbits++;
        size_t need = 0, tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint64_t*)nullptr, (uint64_t*)nullptr, (uint32_t*)nullptr,
                                        (uint32_t*)nullptr, (int)nn, 0, 64, st);
        need = std::max(need, tb);
        cub::DeviceReduce::ReduceByKey(nullptr, tb, sc->key_b.as<uint64_t>(), sc->ukey.as<uint64_t>(), vin,
                                       sc->agg.as<LenAgg>(), sc->runs.as<uint32_t>(), LenAggOp(), (int)nn, st);
        need = std::max(need, tb);
        RGL_TRY(sc->tmp.ensure(need + 256));
    }
    if (n) {
        k_group_keys<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
            n, b->d_intervals + b->block_offsets[0], d_boff, d_tabs, d_tabs + nblk, nblk + 1, d_tabs + 2ull * nblk,
            num_shards, C, m->nb.as<uint64_t>(), (double)bin_size, local ? 1 : 0, sc->key_a.as<uint64_t>(),
            sc->len_a.as<uint32_t>());
        if (local) {
            // sort every block by l_int (every block counts as out of order: lengths come in any order),
            // then the runs of equal keys
            uint32_t* tile_pre = sc->plan.as<uint32_t>();
            uint32_t* chunk_pre = tile_pre + nblk + 1;
            uint32_t* unsorted = chunk_pre + nblk + 1;
            uint32_t* tile_heads = unsorted + nblk;
            uint32_t* tile_off = tile_heads + tiles + 1;
            RGL_CUDA(cudaMemsetAsync(unsorted, 0x01, nblk * 4ull, st));
            block_sort_enqueue(nblk, d_boff, tiles, chunks, sort_passes(max_block), tile_pre, chunk_pre, unsorted,
                               sc->key_a.as<uint64_t>(), sc->len_a.as<uint32_t>(), sc->key_b.as<uint64_t>(),
                               sc->len_b.as<uint32_t>(), tile_off + tiles + 1, st, true);
            if (tiles) {
                k_run_count<<<(unsigned)tiles, kRunThreads, 0, st>>>(nblk, d_boff, tile_pre, sc->key_b.as<uint64_t>(),
                                                                    tile_heads);
                k_scan_small<<<1, 1024, 0, st>>>((uint32_t)tiles, tile_heads, tile_off);
                // run bounds in the sort's scratch keys (free once the blocks are sorted)
                uint32_t* bounds = reinterpret_cast<uint32_t*>(sc->key_a.p);
                k_run_emit<<<(unsigned)tiles, kRunThreads, 0, st>>>(nblk, d_boff, tile_pre, tile_off,
                                                                   sc->key_b.as<uint64_t>(), sc->ukey.as<uint64_t>(),
                                                                   bounds);
                int nsm = 148;
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
                k_run_agg<<<(unsigned)nsm * 8, kRunThreads, 0, st>>>(tile_off + tiles, bounds,
                                                                     sc->len_b.as<uint32_t>(), sc->agg.as<LenAgg>());
                RGL_CUDA(cudaMemcpyAsync(sc->runs.p, tile_off + tiles, 4, cudaMemcpyDeviceToDevice, st));
            } else {
                RGL_CUDA(cudaMemsetAsync(sc->runs.p, 0, 4, st));
            }
        } else {
            size_t tb = sc->tmp.cap;
            RGL_CUDA(cub::DeviceRadixSort::SortPairs(sc->tmp.p, tb, sc->key_a.as<uint64_t>(), sc->key_b.as<uint64_t>(),
                                                     sc->len_a.as<uint32_t>(), sc->len_b.as<uint32_t>(), (int)n, 0,
                                                     std::min(64, 32 + segbits), st));
            tb = sc->tmp.cap;
            RGL_CUDA(cub::DeviceReduce::ReduceByKey(sc->tmp.p, tb, sc->key_b.as<uint64_t>(), sc->ukey.as<uint64_t>(),
                                                    vin, sc->agg.as<LenAgg>(), sc->runs.as<uint32_t>(), LenAggOp(),
                                                    (int)n, st));
        }
    } else {
        RGL_CUDA(cudaMemsetAsync(sc->runs.p, 0, 4, st));
    }
    k_group_finish<<<(unsigned)((nn + 256) / 256), 256, 0, st>>>(
        sc->ukey.as<uint64_t>(), sc->agg.as<LenAgg>(), sc->runs.as<uint32_t>(), rows, C, (double)bin_size,
        m->slot_tab.as<uint32_t>(), lmax, sc->groups.as<QGroupDev>(), d_goff);
    RGL_CUDA(cudaGetLastError());
    *goff_out = d_goff;
    return RGL_OK;
}

namespace rgl {

int batch_pvalues_enqueue(rgl_context* ctx, rgl_moments* m, StatsScratch* sc, const rgl_batch* b,
                          const uint32_t* shard_chrom, uint32_t num_shards, uint32_t bin_size, const uint32_t* d_counts,
                          const uint64_t* d_overlap_bp, double* d_p, double* d_llr, double* d_log_p, uint8_t* d_flags,
                          uint64_t* out_groups) {
    if (!ctx || !m || !b || !d_counts || !d_overlap_bp || !d_p || !d_llr || !d_flags || !bin_size ||
        (num_shards && !shard_chrom))
        return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    bool empty = false;
    uint64_t* d_goff = nullptr;
    RGL_TRY(enqueue_batch_groups(ctx, m, sc, b, shard_chrom, num_shards, bin_size, &empty, &d_goff));
    if (empty) {
        if (out_groups) *out_groups = 0;
        return RGL_OK;
    }
    const uint32_t rows = b->num_rows, D = m->num_sources, C = m->num_chroms;
    cudaStream_t st = context_stream(ctx);
    // the p-value kernel drops groups whose slot lies past the source's table (slot >= tab_len)
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    const uint64_t cells = (uint64_t)rows * D;
    const uint64_t warps = std::min<uint64_t>(cells, (uint64_t)nsm * 64);
    k_pvalues<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(
        rows, D, C, d_counts, reinterpret_cast<const unsigned long long*>(d_overlap_bp), (double)bin_size, d_goff,
        sc->groups.as<QGroupDev>(), m->d_mv, m->coff.as<uint64_t>(), m->stride, m->d_len, d_p, d_llr, d_log_p, d_flags);
    RGL_CUDA(cudaGetLastError());
    if (out_groups) {
        uint64_t ng = 0;
        RGL_CUDA(cudaMemcpyAsync(&ng, d_goff + rows, 8, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaStreamSynchronize(st));
        *out_groups = ng;
    }
    return RGL_OK;
}

}  // namespace rgl

extern "C" {

int rgl_batch_pvalues_device(rgl_context* ctx, rgl_moments* m, const rgl_batch* b, const uint32_t* shard_chrom,
                             uint32_t num_shards, uint32_t bin_size, const uint32_t* d_counts,
                             const uint64_t* d_overlap_bp, double* d_p, double* d_llr, double* d_log_p,
                             uint8_t* d_flags, uint64_t* out_groups) {
    clear_error();
    if (!m) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    return batch_pvalues_enqueue(ctx, m, &m->sc, b, shard_chrom, num_shards, bin_size, d_counts, d_overlap_bp, d_p,
                                 d_llr, d_log_p, d_flags, out_groups);
}

int rgl_batch_query_groups(rgl_context* ctx, rgl_moments* m, const rgl_batch* b, const uint32_t* shard_chrom,
                           uint32_t num_shards, uint32_t bin_size, uint64_t* row_group_offsets, uint32_t* group_chrom,
                           uint64_t* group_l_int, double* group_sum_scale, double* group_sum_scale2,
                           uint64_t* group_count, uint64_t capacity, uint64_t* out_groups) {
    clear_error();
    if (!out_groups) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    bool empty = false;
    uint64_t* d_goff = nullptr;
    RGL_TRY(enqueue_batch_groups(ctx, m, &m->sc, b, shard_chrom, num_shards, bin_size, &empty, &d_goff));
    const uint32_t rows = b->num_rows;
    if (empty) {
        if (row_group_offsets) std::fill(row_group_offsets, row_group_offsets + rows + 1, 0ull);
        *out_groups = 0;
        return RGL_OK;
    }
    cudaStream_t st = context_stream(ctx);
    std::vector<uint64_t> goff(rows + 1ull);
    RGL_CUDA(cudaMemcpyAsync(goff.data(), d_goff, goff.size() * 8, cudaMemcpyDeviceToHost, st));
    RGL_CUDA(cudaStreamSynchronize(st));
    const uint64_t ng = goff[rows];
    *out_groups = ng;
    if (row_group_offsets) std::copy(goff.begin(), goff.end(), row_group_offsets);
    if (!group_chrom && !group_l_int && !group_sum_scale && !group_sum_scale2 && !group_count) return RGL_OK;
    if (ng > capacity) return fail(RGL_ERR_INVALID_ARGUMENT, "group capacity too small");
    std::vector<QGroupDev> g(ng);
    if (ng) RGL_CUDA(cudaMemcpy(g.data(), m->sc.groups.p, ng * sizeof(QGroupDev), cudaMemcpyDeviceToHost));
    for (uint64_t k = 0; k < ng; k++) {
        if (group_chrom) group_chrom[k] = g[k].chrom;
        if (group_l_int) group_l_int[k] = (uint64_t)g[k].l_int;
        if (group_sum_scale) group_sum_scale[k] = g[k].ss;
        if (group_sum_scale2) group_sum_scale2[k] = g[k].ss2;
        if (group_count) group_count[k] = (uint64_t)g[k].count;
    }
    return RGL_OK;
}

}  // extern "C"
