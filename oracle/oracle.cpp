// ============================================================================================
// ORACLE — test infrastructure, NOT product code.
//
// A plain-C++ CPU restatement of the reference crate's (`chuckle`, simondoesstuff/riggle, Rust)
// algorithms for the interval-sweep / sliding-window-moment / analytic-p-value path.  Only the
// tests, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg may load this library, and only
// as the checker (or, for the baseline, as the timed restatement of the reference's CPU path).  The
// product library (riggle_b200/libriggle_b200.so) never links, loads or calls it.
//
// Parity pinning: the reference cannot be compiled here (it is Rust; no cargo/rustc in this image),
// so the restatement is pinned against every known-answer unit test the reference holds for this
// path (src/sweep/query.rs, src/io/jump.rs, src/io/meta.rs, src/io/layer.rs, src/fourier/*.rs,
// src/tasks/query/mod.rs); tests/test_oracle_pins.py ports each one.  The reference's seeded
// integration goldens (tests/integration.rs) depend on rand 0.8.5's StdRng stream (source absent
// from the reference tree) and are therefore "parity unpinned".
//
// Every function cites the reference file:line it restates.  Floating-point code is compiled with
// -ffp-contract=off so that no a*b+c is fused: Rust never contracts, and the f32 depth signal must
// round exactly as the reference's does.
// ============================================================================================
#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// --------------------------------------------------------------------------------------------
// src/io/meta.rs:33-81  — LayerConfig
// --------------------------------------------------------------------------------------------
inline bool is_pow2(uint32_t x) { return x != 0 && (x & (x - 1)) == 0; }

uint32_t layer_for_size(uint32_t min_size, uint32_t gf, uint32_t size) {
    // meta.rs:33-58
    if (size < min_size) return 0;
    if (is_pow2(min_size) && is_pow2(gf) && gf >= 2) {
        uint32_t log2_size = 31u - (uint32_t)__builtin_clz(size);
        uint32_t log2_min = 31u - (uint32_t)__builtin_clz(min_size);
        uint32_t log2_gf = (uint32_t)__builtin_ctz(gf);
        uint32_t diff = log2_size >= log2_min ? log2_size - log2_min : 0;  // saturating_sub
        return diff / log2_gf + 1;
    }
    uint64_t threshold = min_size;
    uint32_t layer = 0;
    // The reference loops forever for min_size == 0 or growth_factor < 2; callers validate first.
    while (threshold <= size) {
        unsigned __int128 t = (unsigned __int128)threshold * gf;
        threshold = t > UINT64_MAX ? UINT64_MAX : (uint64_t)t;  // saturating_mul
        layer++;
    }
    return layer;
}

uint32_t layer_max_size(uint32_t min_size, uint32_t gf, uint32_t layer) {
    // meta.rs:64-73
    uint64_t val = min_size;
    for (uint32_t i = 0; i < layer; i++) {
        unsigned __int128 t = (unsigned __int128)val * gf;
        val = t > UINT64_MAX ? UINT64_MAX : (uint64_t)t;
    }
    return val > UINT32_MAX ? UINT32_MAX : (uint32_t)val;
}

uint32_t tile_size(uint32_t min_size, uint32_t gf, uint32_t layer) {
    // meta.rs:79-81
    uint32_t t = layer_max_size(min_size, gf, layer) / 2;
    return t < 1 ? 1 : t;
}

// --------------------------------------------------------------------------------------------
// src/io/jump.rs
// --------------------------------------------------------------------------------------------
std::vector<uint64_t> build_jump_table(const uint32_t* starts, uint64_t n, uint32_t tile) {
    // jump.rs:66-113.  table[t] = number of intervals with start < t*tile; the reference's
    // sparse-checkpoint/densify construction yields exactly this (its own test at src/io/jump.rs:220-237
    // checks it against partition_point); it is restated here as one sequential pass.
    if (n == 0) return {0};
    uint64_t max_tile = starts[n - 1] / tile;
    std::vector<uint64_t> dense(max_tile + 1, 0);
    uint64_t i = 0;
    for (uint64_t t = 0; t <= max_tile; t++) {
        uint64_t bound = t * (uint64_t)tile;
        while (i < n && (uint64_t)starts[i] < bound) i++;
        dense[t] = i;
    }
    return dense;
}

uint64_t jump_lookup(const uint64_t* table, uint64_t num_tiles, uint32_t tile, uint32_t target) {
    // jump.rs:46-51 (num_tiles >= 1: the reference panics on an empty table)
    uint64_t tile_idx = target / tile;
    uint64_t eff = tile_idx < num_tiles - 1 ? tile_idx : num_tiles - 1;
    return table[eff];
}

// --------------------------------------------------------------------------------------------
// src/sweep/query.rs:84-117 — query_sweep_windowed (identical scan to query_sweep :44-77)
// --------------------------------------------------------------------------------------------
struct Pos {
    uint32_t start, end;
};

struct SweepStats {
    uint64_t candidates = 0;  // positions examined with p.start < q.end (before the break)
    uint64_t hits = 0;        // overlapping pairs
};

void query_sweep_windowed(const Pos* pos, const uint32_t* sids, uint64_t n, uint32_t layer_max,
                          const uint64_t* jt, uint64_t jt_len, uint32_t tile,
                          const uint32_t* q /*start,end,sid triples*/, uint64_t nq, uint32_t q_sid_base,
                          uint32_t cols, uint32_t bin_size, uint32_t* counts, float* overlap,
                          uint64_t* overlap_bp, SweepStats* st) {
    if (nq == 0 || n == 0) return;  // src/sweep/query.rs:94-96
    for (uint64_t k = 0; k < nq; k++) {
        uint32_t qs = q[3 * k], qe = q[3 * k + 1], qsid = q[3 * k + 2];
        uint32_t lo = qs >= layer_max ? qs - layer_max : 0;  // saturating_sub  :141
        uint64_t approx = jump_lookup(jt, jt_len, tile, lo);  // :142
        if (approx > n) approx = n;
        // partition_point(|p| p.start < lo) on pos[approx..]  :143
        uint64_t a = approx, b = n;
        while (a < b) {
            uint64_t m = a + (b - a) / 2;
            if (pos[m].start < lo) a = m + 1; else b = m;
        }
        uint64_t row = (uint64_t)(qsid - q_sid_base);
        for (uint64_t i = a; i < n; i++) {  // :147-158
            const Pos p = pos[i];
            if (p.start >= qe) break;
            if (st) st->candidates++;
            if (p.end > qs) {
                uint32_t d = sids[i];
                counts[row * cols + d] += 1u;  // u32 wrap as in a release build
                uint32_t bp = std::min(qe, p.end) - std::max(qs, p.start);
                float bins = (float)bp / (float)bin_size;
                overlap[row * cols + d] += bins;
                if (overlap_bp) overlap_bp[row * cols + d] += bp;
                if (st) st->hits++;
            }
        }
    }
}

// --------------------------------------------------------------------------------------------
// src/fourier/depth.rs:109-215 — fractional-bin depth signal in f32, reference operation order
// --------------------------------------------------------------------------------------------
void simd_cumsum_f32(float* g, uint64_t n) {
    // depth.rs:143-204
    if (n <= 1) return;
    const uint64_t W = 8;
    uint64_t full = n / W, tail = full * W;
    for (uint64_t c = 0; c < full; c++) {
        uint64_t b = c * W;
        for (uint64_t i = 1; i < W; i++) g[b + i] += g[b + i - 1];
    }
    for (uint64_t i = tail + 1; i < n; i++) g[i] += g[i - 1];
    if (full == 0) return;
    float carry = 0.0f;
    std::vector<float> carries(full);
    for (uint64_t c = 0; c < full; c++) {
        carries[c] = carry;
        carry += g[c * W + W - 1];
    }
    for (uint64_t c = 1; c < full; c++) {
        float off = carries[c];
        for (uint64_t i = 0; i < W; i++) g[c * W + i] = g[c * W + i] + off;
    }
    if (tail < n && carry != 0.0f)
        for (uint64_t i = tail; i < n; i++) g[i] += carry;
}

void build_depth_signal(const uint32_t* starts, const uint32_t* ends, uint64_t n_iv, uint64_t n_bins,
                        uint32_t bin_size, float* g) {
    // build_spikes (depth.rs:206-215): clip coordinates to n_bins*BIN (u32 arithmetic)
    uint32_t max_bp = (uint32_t)n_bins * bin_size;
    std::fill(g, g + n_bins, 0.0f);
    // depth.rs:113-122 — positive spikes in input order
    for (uint64_t i = 0; i < n_iv; i++) {
        uint32_t x = std::min(starts[i], max_bp);
        uint64_t bin = x / bin_size;
        float frac = (float)(x % bin_size) / (float)bin_size;
        if (bin < n_bins) g[bin] += 1.0f - frac;
        if (frac > 0.0f && bin + 1 < n_bins) g[bin + 1] += frac;
    }
    // depth.rs:123-132 — negative spikes in input order
    for (uint64_t i = 0; i < n_iv; i++) {
        uint32_t x = std::min(ends[i], max_bp);
        uint64_t bin = x / bin_size;
        float frac = (float)(x % bin_size) / (float)bin_size;
        if (bin < n_bins) g[bin] -= 1.0f - frac;
        if (frac > 0.0f && bin + 1 < n_bins) g[bin + 1] -= frac;
    }
    simd_cumsum_f32(g, n_bins);  // depth.rs:134
}

// --------------------------------------------------------------------------------------------
// src/fourier/moments.rs — prefix sums, FFT autocorrelation, window moments, L grid
// --------------------------------------------------------------------------------------------
const uint64_t T_THRESHOLD = 100;  // moments.rs:50
const double EPS = 0.01;           // moments.rs:47

uint64_t compact_index(uint64_t l) {
    // moments.rs:58-66
    if (l <= T_THRESHOLD) return l - 1;
    uint64_t k = (uint64_t)(std::log((double)l / (double)T_THRESHOLD) / std::log(1.0 + EPS));
    return T_THRESHOLD + k - 1;
}

std::vector<uint64_t> moment_grid(uint64_t n) {
    // moments.rs:215-247: L = 1..=min(T, N-1) then ceil(T*(1+EPS)^j) by repeated multiplication,
    // deduplicated, while L <= N-1.
    std::vector<uint64_t> ls;
    if (n <= 1) return ls;
    uint64_t max_l = n - 1;
    for (uint64_t l = 1; l <= std::min(T_THRESHOLD, max_l); l++) ls.push_back(l);
    double l_f = (double)T_THRESHOLD;
    uint64_t prev = T_THRESHOLD;
    for (;;) {
        l_f *= 1.0 + EPS;
        uint64_t l = (uint64_t)std::ceil(l_f);
        if (l > max_l) break;
        if (l > prev) {
            ls.push_back(l);
            prev = l;
        }
    }
    return ls;
}

std::vector<double> prefix_sum_f32_to_f64(const float* src, uint64_t n) {
    // moments.rs:262-303 (chunk-of-4 two-pass order)
    std::vector<double> d(n + 1, 0.0);
    const uint64_t W = 4;
    uint64_t chunks = n / W;
    for (uint64_t c = 0; c < chunks; c++) {
        uint64_t b = c * W;
        double g0 = src[b], g1 = src[b + 1], g2 = src[b + 2], g3 = src[b + 3];
        d[b + 1] = g0;
        d[b + 2] = g0 + g1;
        d[b + 3] = g0 + g1 + g2;
        d[b + 4] = g0 + g1 + g2 + g3;
    }
    double carry = 0.0;
    std::vector<double> carries(chunks);
    for (uint64_t c = 0; c < chunks; c++) {
        carries[c] = carry;
        carry += d[c * W + W];
    }
    for (uint64_t c = 1; c < chunks; c++)
        for (uint64_t i = 1; i <= W; i++) d[c * W + i] = d[c * W + i] + carries[c];
    for (uint64_t i = chunks * W; i < n; i++) d[i + 1] = d[i] + (double)src[i];
    return d;
}

std::vector<double> prefix_sum_f64(const std::vector<double>& src, bool square) {
    // moments.rs:306-342 (prefix_sum_f64) and :348-386 (d2_prefix_sum, square=true)
    uint64_t n = src.size();
    std::vector<double> d(n + 1, 0.0);
    const uint64_t W = 4;
    uint64_t chunks = n / W;
    auto v = [&](uint64_t i) { return square ? src[i] * src[i] : src[i]; };
    for (uint64_t c = 0; c < chunks; c++) {
        uint64_t b = c * W;
        double s0 = v(b), s1 = v(b + 1), s2 = v(b + 2), s3 = v(b + 3);
        d[b + 1] = s0;
        d[b + 2] = s0 + s1;
        d[b + 3] = s0 + s1 + s2;
        d[b + 4] = s0 + s1 + s2 + s3;
    }
    double carry = 0.0;
    std::vector<double> carries(chunks);
    for (uint64_t c = 0; c < chunks; c++) {
        carries[c] = carry;
        carry += d[c * W + W];
    }
    for (uint64_t c = 1; c < chunks; c++)
        for (uint64_t i = 1; i <= W; i++) d[c * W + i] = d[c * W + i] + carries[c];
    for (uint64_t i = chunks * W; i < n; i++) d[i + 1] = d[i] + v(i);
    return d;
}

// Radix-2 iterative complex FFT in double precision (the oracle's own; rustfft 6.4.1/realfft 3.5.0
// are not present in this tree — its output is cross-checked against numpy.fft in the tests).
void fft_inplace(std::vector<std::complex<double>>& a, bool inverse) {
    const uint64_t n = a.size();
    for (uint64_t i = 1, j = 0; i < n; i++) {
        uint64_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (uint64_t len = 2; len <= n; len <<= 1) {
        const double ang = 2.0 * M_PI / (double)len * (inverse ? 1.0 : -1.0);
        const uint64_t half = len / 2;
        std::vector<std::complex<double>> w(half);
        for (uint64_t k = 0; k < half; k++) w[k] = std::complex<double>(std::cos(ang * (double)k), std::sin(ang * (double)k));
        for (uint64_t i = 0; i < n; i += len)
            for (uint64_t k = 0; k < half; k++) {
                std::complex<double> u = a[i + k], t = a[i + k + half] * w[k];
                a[i + k] = u + t;
                a[i + k + half] = u - t;
            }
    }
}

std::vector<double> autocorr_via_fft(const std::vector<double>& x) {
    // moments.rs:421-466: zero-pad to next_pow2(2n), |FFT|^2, inverse, scale 1/len, keep n lags.
    uint64_t n = x.size();
    if (n == 0) return {};
    uint64_t len = 1;
    while (len < 2 * n) len <<= 1;
    std::vector<std::complex<double>> a(len, 0.0);
    for (uint64_t i = 0; i < n; i++) a[i] = x[i];
    fft_inplace(a, false);
    for (auto& c : a) c = std::complex<double>(std::norm(c), 0.0);
    fft_inplace(a, true);
    std::vector<double> r(n);
    double scale = 1.0 / (double)len;
    for (uint64_t i = 0; i < n; i++) r[i] = a[i].real() * scale;
    return r;
}

void window_moments(const std::vector<double>& d_ss, const std::vector<double>& d2, const std::vector<double>& r,
                    uint64_t n, uint64_t l, double* mean_out, double* var_out) {
    // moments.rs:392-411
    double n_w = (double)(n - l + 1);
    double sum_f = d_ss[n + 1] - d_ss[l] - d_ss[n - l + 1];
    double r_l = l < r.size() ? r[l] : 0.0;
    double sum_f2 = (d2[n + 1] - d2[l]) + d2[n - l + 1] - 2.0 * r_l;
    double mean = sum_f / n_w;
    double e_f2 = sum_f2 / n_w;
    double var = e_f2 - mean * mean;
    *mean_out = mean;
    *var_out = var > 0.0 ? var : 0.0;
}

// Double-double helpers for the exact moment oracle (TwoSum, Knuth; TwoProduct via fma).
struct DD {
    double hi, lo;
};
inline DD two_sum(double a, double b) {
    double s = a + b, bb = s - a, e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
inline DD dd_add(DD a, DD b) {
    DD s = two_sum(a.hi, b.hi);
    DD t = two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return two_sum(s.hi, s.lo);
}
inline DD dd_neg(DD a) { return {-a.hi, -a.lo}; }
inline DD dd_mul(DD a, DD b) {
    double p = a.hi * b.hi;
    double e = std::fma(a.hi, b.hi, -p);
    e += a.hi * b.lo + a.lo * b.hi;
    return two_sum(p, e);
}
inline DD dd_div_d(DD a, double b) {
    double q1 = a.hi / b;
    DD p = dd_mul({q1, 0.0}, {b, 0.0});
    DD r = dd_add(a, dd_neg(p));
    double q2 = r.hi / b;
    return two_sum(q1, q2);
}

// --------------------------------------------------------------------------------------------
// src/fourier/stats.rs:34-126
// --------------------------------------------------------------------------------------------
double erfc_as(double x) {
    // stats.rs:116-126 (Abramowitz & Stegun 7.1.26 as written in the reference)
    if (x < 0.0) return 2.0 - erfc_as(-x);
    double t = 1.0 / (1.0 + 0.3275911 * x);
    double p = t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
    return p * std::exp(-x * x);
}

bool nb_llr(double mu, double var, double observed, double* out) {
    // stats.rs:101-113
    if (mu <= 0.0 || var <= mu) return false;
    double r = mu * mu / (var - mu);
    double p = mu / var;
    double p_o = r / (r + observed);
    if (!(0.0 < p && p < 1.0 && 0.0 < p_o && p_o < 1.0)) return false;
    double theta = std::log((1.0 - p_o) / (1.0 - p));
    *out = observed * theta + r * std::log(p_o / p);
    return true;
}

bool poisson_llr(double mu, double observed, double* out) {
    // stats.rs:93-98
    if (mu <= 0.0 || observed <= 0.0) return false;
    *out = observed * std::log(observed / mu) - (observed - mu);
    return true;
}

}  // namespace

// ============================================================================================
// C ABI of the oracle (loaded with ctypes by the tests and the CPU-baseline leg only)
// ============================================================================================
extern "C" {

uint32_t orc_layer_for_size(uint32_t min_size, uint32_t gf, uint32_t size) { return layer_for_size(min_size, gf, size); }
uint32_t orc_layer_max_size(uint32_t min_size, uint32_t gf, uint32_t layer) { return layer_max_size(min_size, gf, layer); }
uint32_t orc_tile_size(uint32_t min_size, uint32_t gf, uint32_t layer) { return tile_size(min_size, gf, layer); }

// jump.rs:66-113; returns the table length, writes min(len, cap) entries.
uint64_t orc_build_jump_table(const uint32_t* starts, uint64_t n, uint32_t tile, uint64_t* out, uint64_t cap) {
    auto t = build_jump_table(starts, n, tile);
    for (uint64_t i = 0; i < t.size() && i < cap; i++) out[i] = t[i];
    return t.size();
}

// jump.rs:135-169: merged[t] = old[t] + new_local[t] (missing entries read as 0).
uint64_t orc_extend_jump_table(const uint64_t* old_t, uint64_t n_old, const uint32_t* new_starts, uint64_t n_new,
                               uint32_t tile, uint64_t* out, uint64_t cap) {
    if (n_new == 0) {
        for (uint64_t i = 0; i < n_old && i < cap; i++) out[i] = old_t[i];
        return n_old;
    }
    auto nl = build_jump_table(new_starts, n_new, tile);
    uint64_t len = std::max<uint64_t>(n_old, nl.size());
    for (uint64_t t = 0; t < len && t < cap; t++) out[t] = (t < n_old ? old_t[t] : 0) + (t < nl.size() ? nl[t] : 0);
    return len;
}

uint64_t orc_jump_lookup(const uint64_t* table, uint64_t n, uint32_t tile, uint32_t target) {
    return jump_lookup(table, n, tile, target);
}

// layer.rs:135-199 — reverse co-merge of new_sorted into an existing sorted layer (in memory).
// out_pos/out_sid hold n_old+n_new entries; old entries win ties (>=), as in the reference.
void orc_extend_layer(const uint32_t* old_pos, const uint32_t* old_sid, uint64_t n_old, const uint32_t* new_ivs,
                      uint64_t n_new, uint32_t* out_pos, uint32_t* out_sid) {
    uint64_t total = n_old + n_new;
    std::vector<uint32_t> p(2 * total), s(total);
    for (uint64_t i = 0; i < n_old; i++) {
        p[2 * i] = old_pos[2 * i];
        p[2 * i + 1] = old_pos[2 * i + 1];
        s[i] = old_sid[i];
    }
    uint64_t old_ptr = n_old, new_ptr = n_new, out_ptr = total;
    while (old_ptr > 0 && new_ptr > 0) {
        out_ptr--;
        if (p[2 * (old_ptr - 1)] >= new_ivs[3 * (new_ptr - 1)]) {
            p[2 * out_ptr] = p[2 * (old_ptr - 1)];
            p[2 * out_ptr + 1] = p[2 * (old_ptr - 1) + 1];
            s[out_ptr] = s[old_ptr - 1];
            old_ptr--;
        } else {
            p[2 * out_ptr] = new_ivs[3 * (new_ptr - 1)];
            p[2 * out_ptr + 1] = new_ivs[3 * (new_ptr - 1) + 1];
            s[out_ptr] = new_ivs[3 * (new_ptr - 1) + 2];
            new_ptr--;
        }
    }
    while (new_ptr > 0) {
        out_ptr--;
        p[2 * out_ptr] = new_ivs[3 * (new_ptr - 1)];
        p[2 * out_ptr + 1] = new_ivs[3 * (new_ptr - 1) + 1];
        s[out_ptr] = new_ivs[3 * (new_ptr - 1) + 2];
        new_ptr--;
    }
    std::memcpy(out_pos, p.data(), 8 * total);
    std::memcpy(out_sid, s.data(), 4 * total);
}

// src/sweep/query.rs:84-117 on one layer.  counts/overlap are rows x cols row-major, row = qsid - base.
void orc_query_sweep_windowed(const uint32_t* pos, const uint32_t* sids, uint64_t n, uint32_t layer_max,
                              const uint64_t* jt, uint64_t jt_len, uint32_t tile, const uint32_t* q, uint64_t nq,
                              uint32_t q_sid_base, uint32_t cols, uint32_t bin_size, uint32_t* counts,
                              float* overlap) {
    query_sweep_windowed(reinterpret_cast<const Pos*>(pos), sids, n, layer_max, jt, jt_len, tile, q, nq, q_sid_base,
                         cols, bin_size, counts, overlap, nullptr, nullptr);
}

// One (shard, layer) of an in-memory index, in the reference's on-disk layout:
// pos = layer_K.pos ((start,end) u32 pairs sorted by start), sid = layer_K.sid, jump = layer_K.idx.
typedef struct {
    uint32_t shard;
    uint32_t layer;
    uint64_t count;
    const uint32_t* pos;
    const uint32_t* sid;
    const uint64_t* jump;  // NULL: built with build_jump_table (as a freshly written layer has)
    uint64_t jump_len;
} orc_layer;

// Queries of one shard: `count` (start,end,qsid) triples, any order (the driver sorts them).
typedef struct {
    uint32_t shard;
    uint64_t count;
    const uint32_t* ivs;
} orc_qshard;

// Restatement of query_database's counting path (src/tasks/query/mod.rs:182-307) over an in-memory
// index.  mode 0 = the reference's parallel structure (rayon over windows of 64 query rows; shards
// serial, mod.rs:193,243-278); mode 1 = labelled "query-block parallel" variant (each window's
// queries split over `threads` workers; not the reference's structure).  Outputs are dense
// rows x num_sources: counts (u32, wrapping), overlap_f32 (the reference's f32 bins, summed in this
// restatement's fixed shard order; the reference's HashMap shard order makes its own value
// order-dependent) and overlap_bp (exact u64 base pairs).  stats[0] = candidate positions scanned,
// stats[1] = overlapping pairs, stats[2] = union of candidate ranges over all (shard, layer)
// ("DB intervals swept"), stats[3] = query intervals.
int orc_query_database(uint32_t min_size, uint32_t gf, uint32_t num_sources, uint32_t bin_size, uint32_t n_layers,
                       const orc_layer* layers, uint32_t n_qshards, const orc_qshard* qshards, uint32_t rows,
                       int threads, int mode, uint32_t* counts, float* overlap_f32, uint64_t* overlap_bp,
                       uint64_t* stats) {
    const uint64_t cells = (uint64_t)rows * num_sources;
    std::fill(counts, counts + cells, 0u);
    if (overlap_f32) std::fill(overlap_f32, overlap_f32 + cells, 0.0f);
    if (overlap_bp) std::fill(overlap_bp, overlap_bp + cells, 0ull);
    uint64_t st_cand = 0, st_hits = 0, st_union = 0, st_q = 0;
    if (threads < 1) threads = 1;
    const uint64_t WIN = 64;  // SWEEP_WINDOW_SIZE, mod.rs:23

    // shards in ascending index order
    std::vector<const orc_qshard*> qs_sorted;
    for (uint32_t i = 0; i < n_qshards; i++) qs_sorted.push_back(&qshards[i]);
    std::stable_sort(qs_sorted.begin(), qs_sorted.end(), [](auto a, auto b) { return a->shard < b->shard; });

    for (const orc_qshard* qsh : qs_sorted) {
        if (qsh->count == 0) continue;
        // sort by (sid, start): mod.rs:202
        std::vector<uint32_t> sq(qsh->ivs, qsh->ivs + 3 * qsh->count);
        std::vector<uint64_t> order(qsh->count);
        for (uint64_t i = 0; i < qsh->count; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) {
            uint32_t sa = qsh->ivs[3 * a + 2], sb = qsh->ivs[3 * b + 2];
            if (sa != sb) return sa < sb;
            return qsh->ivs[3 * a] < qsh->ivs[3 * b];
        });
        for (uint64_t i = 0; i < qsh->count; i++)
            for (int c = 0; c < 3; c++) sq[3 * i + c] = qsh->ivs[3 * order[i] + c];
        st_q += qsh->count;

        // layers of this shard in layer order, non-empty only (mod.rs:205-236)
        struct L {
            const orc_layer* l;
            uint32_t max_size, tile;
            std::vector<uint64_t> jt_own;
            const uint64_t* jt;
            uint64_t jt_len;
        };
        std::vector<L> ls;
        for (uint32_t i = 0; i < n_layers; i++)
            if (layers[i].shard == qsh->shard && layers[i].count > 0) {
                L x;
                x.l = &layers[i];
                x.max_size = layer_max_size(min_size, gf, layers[i].layer);
                x.tile = tile_size(min_size, gf, layers[i].layer);
                ls.push_back(x);
            }
        std::sort(ls.begin(), ls.end(), [](const L& a, const L& b) { return a.l->layer < b.l->layer; });
        if (ls.empty()) continue;
        for (auto& x : ls) {
            if (x.l->jump) {
                x.jt = x.l->jump;
                x.jt_len = x.l->jump_len;
            } else {
                std::vector<uint32_t> st(x.l->count);
                for (uint64_t i = 0; i < x.l->count; i++) st[i] = x.l->pos[2 * i];
                x.jt_own = build_jump_table(st.data(), st.size(), x.tile);
                x.jt = x.jt_own.data();
                x.jt_len = x.jt_own.size();
            }
        }

        // union of candidate ranges per layer over all queries of the shard (metric definition)
        for (auto& x : ls) {
            const Pos* pos = reinterpret_cast<const Pos*>(x.l->pos);
            uint64_t n = x.l->count;
            std::vector<std::pair<uint64_t, uint64_t>> rg;
            for (uint64_t i = 0; i < qsh->count; i++) {
                uint32_t qs0 = sq[3 * i], qe0 = sq[3 * i + 1];
                uint32_t lo = qs0 >= x.max_size ? qs0 - x.max_size : 0;
                uint64_t a = std::partition_point(pos, pos + n, [&](const Pos& p) { return p.start < lo; }) - pos;
                uint64_t b = std::partition_point(pos, pos + n, [&](const Pos& p) { return p.start < qe0; }) - pos;
                if (b > a) rg.push_back({a, b});
            }
            std::sort(rg.begin(), rg.end());
            uint64_t cur_lo = 0, cur_hi = 0;
            bool open = false;
            for (auto& r : rg) {
                if (!open || r.first > cur_hi) {
                    if (open) st_union += cur_hi - cur_lo;
                    cur_lo = r.first;
                    cur_hi = r.second;
                    open = true;
                } else
                    cur_hi = std::max(cur_hi, r.second);
            }
            if (open) st_union += cur_hi - cur_lo;
        }

        // windows of 64 Q_SID rows (mod.rs:243-278)
        uint64_t n_windows = (rows + WIN - 1) / WIN;
        struct WinOut {
            std::vector<uint32_t> c;
            std::vector<float> o;
            std::vector<uint64_t> bp;
            SweepStats st;
        };
        auto window_range = [&](uint64_t w, uint64_t* lo, uint64_t* hi) {
            uint32_t qlo = (uint32_t)(w * WIN), qhi = (uint32_t)std::min<uint64_t>((w + 1) * WIN, rows);
            uint64_t a = 0, b = qsh->count;
            while (a < b) { uint64_t m = (a + b) / 2; if (sq[3 * m + 2] < qlo) a = m + 1; else b = m; }
            *lo = a;
            a = 0; b = qsh->count;
            while (a < b) { uint64_t m = (a + b) / 2; if (sq[3 * m + 2] < qhi) a = m + 1; else b = m; }
            *hi = a;
        };
        auto run_block = [&](uint64_t w, uint64_t qlo_i, uint64_t qhi_i, WinOut& out) {
            uint32_t base = (uint32_t)(w * WIN);
            uint32_t wrows = (uint32_t)(std::min<uint64_t>((w + 1) * WIN, rows) - w * WIN);
            out.c.assign((uint64_t)wrows * num_sources, 0u);
            out.o.assign((uint64_t)wrows * num_sources, 0.0f);
            out.bp.assign((uint64_t)wrows * num_sources, 0ull);
            for (auto& x : ls)
                query_sweep_windowed(reinterpret_cast<const Pos*>(x.l->pos), x.l->sid, x.l->count, x.max_size, x.jt,
                                     x.jt_len, x.tile, sq.data() + 3 * qlo_i, qhi_i - qlo_i, base, num_sources,
                                     bin_size, out.c.data(), out.o.data(), out.bp.data(), &out.st);
        };
        auto merge = [&](uint64_t w, WinOut& out) {  // add_submatrix_rows, mod.rs:280-285
            uint64_t off = w * WIN * num_sources;
            for (uint64_t i = 0; i < out.c.size(); i++) {
                counts[off + i] += out.c[i];
                if (overlap_f32) overlap_f32[off + i] += out.o[i];
                if (overlap_bp) overlap_bp[off + i] += out.bp[i];
            }
            st_cand += out.st.candidates;
            st_hits += out.st.hits;
        };

        if (mode == 0) {
            std::vector<WinOut> outs(n_windows);
            std::atomic<uint64_t> next{0};
            auto worker = [&]() {
                for (;;) {
                    uint64_t w = next.fetch_add(1);
                    if (w >= n_windows) break;
                    uint64_t lo, hi;
                    window_range(w, &lo, &hi);
                    run_block(w, lo, hi, outs[w]);
                }
            };
            int nt = (int)std::min<uint64_t>((uint64_t)threads, n_windows);
            std::vector<std::thread> th;
            for (int t = 1; t < nt; t++) th.emplace_back(worker);
            worker();
            for (auto& t : th) t.join();
            for (uint64_t w = 0; w < n_windows; w++) merge(w, outs[w]);
        } else {
            // query-block parallel: each window's query slice split across threads
            for (uint64_t w = 0; w < n_windows; w++) {
                uint64_t lo, hi;
                window_range(w, &lo, &hi);
                uint64_t nq = hi - lo;
                int nt = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)threads, nq));
                std::vector<WinOut> outs(nt);
                std::vector<std::thread> th;
                for (int t = 0; t < nt; t++) {
                    uint64_t a = lo + nq * t / nt, b = lo + nq * (t + 1) / nt;
                    th.emplace_back([&, t, a, b]() { run_block(w, a, b, outs[t]); });
                }
                for (auto& t : th) t.join();
                for (int t = 0; t < nt; t++) merge(w, outs[t]);
            }
        }
    }
    if (stats) {
        stats[0] = st_cand;
        stats[1] = st_hits;
        stats[2] = st_union;
        stats[3] = st_q;
    }
    return 0;
}

// Brute-force O(Nq * Nd) pair oracle of the same predicate (src/sweep/query.rs:98-108 with the layer
// look-back bound) — independent of jump tables and scans; small cases only.
void orc_bruteforce_counts(uint32_t min_size, uint32_t gf, uint32_t num_sources, uint32_t n_layers,
                           const orc_layer* layers, uint32_t n_qshards, const orc_qshard* qshards, uint32_t rows,
                           uint32_t* counts, uint64_t* overlap_bp) {
    std::fill(counts, counts + (uint64_t)rows * num_sources, 0u);
    std::fill(overlap_bp, overlap_bp + (uint64_t)rows * num_sources, 0ull);
    for (uint32_t s = 0; s < n_qshards; s++)
        for (uint32_t l = 0; l < n_layers; l++) {
            if (layers[l].shard != qshards[s].shard) continue;
            uint32_t mx = layer_max_size(min_size, gf, layers[l].layer);
            for (uint64_t i = 0; i < qshards[s].count; i++) {
                uint32_t qs = qshards[s].ivs[3 * i], qe = qshards[s].ivs[3 * i + 1], qsid = qshards[s].ivs[3 * i + 2];
                uint32_t lo = qs >= mx ? qs - mx : 0;
                for (uint64_t j = 0; j < layers[l].count; j++) {
                    uint32_t ds = layers[l].pos[2 * j], de = layers[l].pos[2 * j + 1];
                    if (ds >= lo && ds < qe && de > qs) {
                        uint64_t cell = (uint64_t)qsid * num_sources + layers[l].sid[j];
                        counts[cell] += 1u;
                        overlap_bp[cell] += std::min(qe, de) - std::max(qs, ds);
                    }
                }
            }
        }
}

// Restatement of `--intervals` mode: query_sweep_pairs (src/sweep/query.rs:11-41) driven as
// collect_interval_pairs (src/tasks/query/intervals.rs:16-112): per shard (ascending index here;
// a HashMap order in the reference), per layer in ascending index, the shard's queries sorted by
// start (voracious_sort keys an Interval by its start, src/core/mod.rs:36-42), and for every query
// the layer's positions from the jump-table seek + partition point while p.start < q.end, emitting
// the pairs with p.end > q.start.  Record: q.start, q.end, d.start, d.end, q.sid (row), d.sid,
// shard, intersection bp.  Returns the number of pairs; writes at most `cap`.
uint64_t orc_query_pairs(uint32_t min_size, uint32_t gf, uint32_t n_layers, const orc_layer* layers,
                         uint32_t n_qshards, const orc_qshard* qshards, uint32_t* out, uint64_t cap) {
    uint64_t np = 0;
    std::vector<const orc_qshard*> qs_sorted;
    for (uint32_t i = 0; i < n_qshards; i++) qs_sorted.push_back(&qshards[i]);
    std::stable_sort(qs_sorted.begin(), qs_sorted.end(), [](auto a, auto b) { return a->shard < b->shard; });
    for (const orc_qshard* qsh : qs_sorted) {
        if (qsh->count == 0) continue;
        std::vector<uint64_t> order(qsh->count);
        for (uint64_t i = 0; i < qsh->count; i++) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](uint64_t a, uint64_t b) { return qsh->ivs[3 * a] < qsh->ivs[3 * b]; });
        std::vector<const orc_layer*> ls;
        for (uint32_t l = 0; l < n_layers; l++)
            if (layers[l].shard == qsh->shard && layers[l].count) ls.push_back(&layers[l]);
        std::stable_sort(ls.begin(), ls.end(), [](auto a, auto b) { return a->layer < b->layer; });
        for (const orc_layer* L : ls) {
            const uint32_t mx = layer_max_size(min_size, gf, L->layer);
            const uint32_t tile = tile_size(min_size, gf, L->layer);
            std::vector<uint64_t> own;
            const uint64_t* jt = L->jump;
            uint64_t jt_len = L->jump_len;
            if (!jt) {
                std::vector<uint32_t> st(L->count);
                for (uint64_t i = 0; i < L->count; i++) st[i] = L->pos[2 * i];
                own = build_jump_table(st.data(), L->count, tile);
                jt = own.data();
                jt_len = own.size();
            }
            const Pos* pos = reinterpret_cast<const Pos*>(L->pos);
            for (uint64_t k : order) {
                const uint32_t qs = qsh->ivs[3 * k], qe = qsh->ivs[3 * k + 1], qsid = qsh->ivs[3 * k + 2];
                const uint32_t lo = qs >= mx ? qs - mx : 0;  // query.rs:23
                uint64_t a = jump_lookup(jt, jt_len, tile, lo);
                if (a > L->count) a = L->count;
                uint64_t b = L->count;
                while (a < b) {  // partition_point(|p| p.start < lo), query.rs:25
                    const uint64_t m = a + (b - a) / 2;
                    if (pos[m].start < lo) a = m + 1; else b = m;
                }
                for (uint64_t i = a; i < L->count; i++) {  // query.rs:28-39
                    const Pos p = pos[i];
                    if (p.start >= qe) break;
                    if (p.end > qs) {
                        if (np < cap && out) {
                            uint32_t* r = out + 8 * np;
                            r[0] = qs;
                            r[1] = qe;
                            r[2] = p.start;
                            r[3] = p.end;
                            r[4] = qsid;
                            r[5] = L->sid[i];
                            r[6] = qsh->shard;
                            r[7] = std::min(qe, p.end) - std::max(qs, p.start);
                        }
                        np++;
                    }
                }
            }
        }
    }
    return np;
}

// ---- fourier ------------------------------------------------------------------------------
void orc_simd_cumsum_f32(float* g, uint64_t n) { simd_cumsum_f32(g, n); }

void orc_build_depth_signal(const uint32_t* starts, const uint32_t* ends, uint64_t n_iv, uint64_t n_bins,
                            uint32_t bin_size, float* g) {
    build_depth_signal(starts, ends, n_iv, n_bins, bin_size, g);
}

uint64_t orc_compact_index(uint64_t l) { return compact_index(l); }

uint64_t orc_moment_grid(uint64_t n_bins, uint64_t* out, uint64_t cap) {
    auto g = moment_grid(n_bins);
    for (uint64_t i = 0; i < g.size() && i < cap; i++) out[i] = g[i];
    return g.size();
}

void orc_autocorr_fft(const double* x, uint64_t n, double* r) {
    std::vector<double> v(x, x + n);
    auto out = autocorr_via_fft(v);
    std::copy(out.begin(), out.end(), r);
}

void orc_prefix_sum_f32_to_f64(const float* src, uint64_t n, double* out) {
    auto d = prefix_sum_f32_to_f64(src, n);
    std::copy(d.begin(), d.end(), out);
}

void orc_d2_prefix_sum(const double* src, uint64_t n, double* out) {
    std::vector<double> v(src, src + n);
    auto d = prefix_sum_f64(v, true);
    std::copy(d.begin(), d.end(), out);
}

void orc_window_moments_from_dstar(const double* d_star, uint64_t n /*bins*/, uint64_t l, double* mean, double* var) {
    // test hook for moments.rs:511-562: d_star has n+1 entries
    std::vector<double> ds(d_star, d_star + n + 1);
    auto d_ss = prefix_sum_f64(ds, false);
    auto d2 = prefix_sum_f64(ds, true);
    auto r = autocorr_via_fft(ds);
    window_moments(d_ss, d2, r, n, l, mean, var);
}

// moments_from_signal (moments.rs:192-254) with f64 outputs; returns the number of grid entries.
// mean_var_f32: 2*entries floats as the store keeps them; mean_f64/var_f64: the unrounded values.
uint64_t orc_moments_from_signal(const float* g, uint64_t n, float* mean_var_f32, double* mean_f64, double* var_f64) {
    if (n <= 1) return 0;
    auto d_star = prefix_sum_f32_to_f64(g, n);
    auto d_ss = prefix_sum_f64(d_star, false);
    auto d2 = prefix_sum_f64(d_star, true);
    auto r = autocorr_via_fft(d_star);
    auto grid = moment_grid(n);
    for (uint64_t i = 0; i < grid.size(); i++) {
        double m, v;
        window_moments(d_ss, d2, r, n, grid[i], &m, &v);
        if (mean_var_f32) {
            mean_var_f32[2 * i] = (float)m;
            mean_var_f32[2 * i + 1] = (float)v;
        }
        if (mean_f64) mean_f64[i] = m;
        if (var_f64) var_f64[i] = v;
    }
    return grid.size();
}

// "Exact" window moments of the same f32 signal for the error reports: for each requested L, the
// mean and variance of the N-L+1 window sums computed directly in double-double (two-pass), which
// has no cancellation against autocorrelation terms.  O(N) per L.
void orc_moments_exact(const float* g, uint64_t n, const uint64_t* ls, uint64_t n_l, double* mean_out, double* var_out,
                       int threads) {
    std::vector<DD> ds(n + 1);
    ds[0] = {0.0, 0.0};
    for (uint64_t i = 0; i < n; i++) ds[i + 1] = dd_add(ds[i], {(double)g[i], 0.0});
    if (threads < 1) threads = 1;
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            uint64_t k = next.fetch_add(1);
            if (k >= n_l) break;
            uint64_t l = ls[k];
            uint64_t nw = n - l + 1;
            DD s = {0.0, 0.0};
            for (uint64_t j = 0; j < nw; j++) s = dd_add(s, dd_add(ds[j + l], dd_neg(ds[j])));
            DD mean = dd_div_d(s, (double)nw);
            DD s2 = {0.0, 0.0};
            for (uint64_t j = 0; j < nw; j++) {
                DD f = dd_add(dd_add(ds[j + l], dd_neg(ds[j])), dd_neg(mean));
                s2 = dd_add(s2, dd_mul(f, f));
            }
            DD var = dd_div_d(s2, (double)nw);
            mean_out[k] = mean.hi + mean.lo;
            var_out[k] = var.hi + var.lo;
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < threads; t++) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
}

// ---- stats --------------------------------------------------------------------------------
double orc_erfc(double x) { return erfc_as(x); }
int orc_nb_llr(double mu, double var, double obs, double* out) { return nb_llr(mu, var, obs, out) ? 1 : 0; }
int orc_poisson_llr(double mu, double obs, double* out) { return poisson_llr(mu, obs, out) ? 1 : 0; }

// build_query_chrom_data (moments.rs:138-177) for one chromosome's lengths: groups by
// l_int = max(ceil(l),1) over ascending l = (e-s)/BIN.  Returns the number of groups.
uint64_t orc_query_groups(const uint32_t* starts, const uint32_t* ends, uint64_t n, uint32_t bin_size,
                          uint64_t* l_int, double* sum_scale, double* sum_scale2, uint64_t* count) {
    std::vector<double> lengths(n);
    for (uint64_t i = 0; i < n; i++) lengths[i] = (double)(ends[i] - starts[i]) / (double)bin_size;
    std::sort(lengths.begin(), lengths.end());
    uint64_t ng = 0, i = 0;
    auto lint_of = [](double l) { uint64_t c = (uint64_t)std::ceil(l); return c < 1 ? (uint64_t)1 : c; };
    while (i < n) {
        double l = lengths[i];
        uint64_t li = lint_of(l);
        double s0 = l / (double)li;
        double ss = s0, ss2 = s0 * s0;
        uint64_t c = 1;
        i++;
        while (i < n && lint_of(lengths[i]) == li) {
            double s = lengths[i] / (double)li;
            ss += s;
            ss2 += s * s;
            c++;
            i++;
        }
        l_int[ng] = li;
        sum_scale[ng] = ss;
        sum_scale2[ng] = ss2;
        count[ng] = c;
        ng++;
    }
    return ng;
}

// compute_analytic_stats (stats.rs:34-88) with the moment-store lookup of
// momentstore.rs:66-79 (compact_index slot, bounds on l_int and table length).
// Query side: n_qc chromosomes; chromosome k has chrom id qc_chrom[k] and groups
// [qc_goff[k], qc_goff[k+1]).  DB side (one source): for chrom id c, db_nbins[c] (0 = absent) and
// db_len[c] entries at db_mv + 2*db_off[c].  Returns 0 when no chromosome/group is shared (None),
// else 1 with *p, *llr, *has_llr.
int orc_analytic_stats(uint32_t n_qc, const uint32_t* qc_chrom, const uint64_t* qc_goff, const uint64_t* g_lint,
                       const double* g_ss, const double* g_ss2, const uint64_t* g_count, const uint64_t* db_nbins,
                       const uint64_t* db_off, const uint64_t* db_len, const float* db_mv, double observed,
                       double* p_out, double* llr_out, int* has_llr) {
    double mu_total = 0.0, var_total = 0.0, mu_raw = 0.0;
    bool any = false;
    for (uint32_t k = 0; k < n_qc; k++) {
        uint32_t c = qc_chrom[k];
        if (db_nbins[c] == 0) continue;  // resolve_chrom -> None
        for (uint64_t gi = qc_goff[k]; gi < qc_goff[k + 1]; gi++) {
            uint64_t l = g_lint[gi];
            if (l == 0 || l >= db_nbins[c]) continue;
            uint64_t base = compact_index(l) * 2;
            if (base + 1 >= 2 * db_len[c]) continue;
            double mean = (double)db_mv[2 * db_off[c] + base], var = (double)db_mv[2 * db_off[c] + base + 1];
            mu_total += mean * g_ss[gi];
            var_total += var * g_ss2[gi];
            mu_raw += mean / (double)l * (double)g_count[gi];
            any = true;
        }
    }
    if (!any) return 0;
    double llr = 0.0;
    bool ok;
    if (var_total > mu_total)
        ok = nb_llr(mu_total, var_total, observed, &llr);
    else {
        double eff = mu_raw > 0.0 ? mu_total / mu_raw : 1.0;
        ok = poisson_llr(mu_raw, observed / eff, &llr);
    }
    double p = 1.0;
    if (ok && llr > 0.0) {
        double tail = erfc_as(std::sqrt(llr)) * 0.5;
        p = observed >= mu_total ? tail : 1.0 - tail;
    }
    *p_out = p;
    *llr_out = ok ? llr : 0.0;
    *has_llr = ok ? 1 : 0;
    return 1;
}

// ln of the right-tail p-value as the reference evaluates it (stats.rs:79-85, 116-126), in a form
// that never underflows: ln(0.5*t*poly(t)) - x*x for enrichment, log1p(-tail) for depletion.
double orc_log_p(double llr, int has_llr, double observed, double mu_total) {
    if (!has_llr || !(llr > 0.0)) return 0.0;
    double x = std::sqrt(llr);
    double t = 1.0 / (1.0 + 0.3275911 * x);
    double poly = t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
    double ln_tail = std::log(0.5 * poly) + (-x * x);
    if (observed >= mu_total) return ln_tail;
    return std::log1p(-std::exp(ln_tail));
}

}  // extern "C"
