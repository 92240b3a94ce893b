// Seeded synthetic workloads for the CPU side of the benchmark (test infrastructure, like the rest
// of oracle/): the same interval model and the same bits as the library's generator, written
// independently so that the CPU reference arm builds its database layers and query files without
// loading the GPU library.  tests/test_oracle_pins.py checks the two generators agree bit for bit.
//
// Streams: SplitMix64 (Steele, Lea & Flood, OOPSLA 2014; finaliser constants as published by Vigna)
// used as a counter-based generator: draw i of stream k is mix64(k + (i + 1) * golden ratio).  An
// interval uses four draws: broad-or-not, length quantile, start, hot-spot-or-not.  Lengths come from
// 65537-point quantile tables (LogNormal(ln 500, 1) clipped to [20, 100000] bp; LogUniform[10k, 1M]
// for broad intervals) with 16-bit integer interpolation; starts are a 32x32-bit multiply-high.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

inline uint64_t sm_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t sm_draw(uint64_t key, uint64_t i) { return sm_mix(key + (i + 1) * 0x9E3779B97F4A7C15ull); }
inline uint64_t sm_key(uint64_t seed, uint64_t file, uint64_t chrom) {
    return sm_mix(sm_mix(seed * 0xD1B54A32D192ED03ull + file) ^ (chrom * 0x8CB92BA72F3D8DD7ull + 0x632BE59BD9B4E019ull));
}
inline uint32_t mul_hi(uint64_t u, uint32_t range) { return (uint32_t)(((u >> 32) * (uint64_t)range) >> 32); }
inline uint32_t table_at(const std::vector<uint32_t>& T, uint64_t u) {
    const uint32_t i = (uint32_t)(u >> 48), f = (uint32_t)((u >> 32) & 0xFFFFu);
    const uint32_t a = T[i], b = T[i + 1];
    return a + (uint32_t)(((uint64_t)(b - a) * f) >> 16);
}

// Standard normal quantile: P. J. Acklam's rational approximation (2003) with one Halley step on
// erfc, the published coefficients.
double normal_quantile(double p) {
    static const double A[] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                               1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double B[] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                               6.680131188771972e+01, -1.328068155288572e+01};
    static const double Cc[] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double Dd[] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    const double lo = 0.02425;
    double x;
    if (p < lo || p > 1 - lo) {
        const double q = std::sqrt(-2 * std::log(p < lo ? p : 1 - p));
        const double v = (((((Cc[0] * q + Cc[1]) * q + Cc[2]) * q + Cc[3]) * q + Cc[4]) * q + Cc[5]) /
                         ((((Dd[0] * q + Dd[1]) * q + Dd[2]) * q + Dd[3]) * q + 1);
        x = p < lo ? v : -v;
    } else {
        const double q = p - 0.5, r = q * q;
        x = (((((A[0] * r + A[1]) * r + A[2]) * r + A[3]) * r + A[4]) * r + A[5]) * q /
            (((((B[0] * r + B[1]) * r + B[2]) * r + B[3]) * r + B[4]) * r + 1);
    }
    const double e = 0.5 * std::erfc(-x / std::sqrt(2.0)) - p;
    const double u = e * std::sqrt(2 * M_PI) * std::exp(x * x / 2);
    return x - u / (1 + x * u / 2);
}

struct Tables {
    std::vector<uint32_t> narrow, broad;
    Tables() : narrow(65537), broad(65537) {
        for (int k = 0; k <= 65536; k++) {
            double v = k == 0 ? 20.0 : k == 65536 ? 100000.0 : std::exp(std::log(500.0) + normal_quantile(k / 65536.0));
            narrow[k] = (uint32_t)std::llround(std::min(100000.0, std::max(20.0, v)));
            broad[k] = (uint32_t)std::llround(std::min(1000000.0, 10000.0 * std::pow(100.0, k / 65536.0)));
        }
    }
};
const Tables& tables() {
    static const Tables t;
    return t;
}

struct Model {
    uint64_t seed, broad_thr, hot_thr;
    uint32_t num_hotspots, sid_base;
};

void one_interval(const Model& m, uint32_t file, uint32_t chrom, uint32_t chrom_len, uint64_t i, uint32_t* s,
                  uint32_t* e) {
    const Tables& T = tables();
    const uint64_t key = sm_key(m.seed + file, file, chrom);
    const uint64_t u0 = sm_draw(key, 4 * i), u1 = sm_draw(key, 4 * i + 1), u2 = sm_draw(key, 4 * i + 2),
                   u3 = sm_draw(key, 4 * i + 3);
    const bool broad = (u0 >> 11) < m.broad_thr;
    const bool hot = !broad && m.num_hotspots > 0 && (u3 >> 11) < m.hot_thr;
    uint32_t len = table_at(broad ? T.broad : T.narrow, u1);
    if (len >= chrom_len) len = chrom_len - 1;
    uint32_t start;
    if (hot && chrom_len > 2000000u) {
        const uint64_t spots = sm_key(m.seed ^ 0x5151515151515151ull, 0xFFFFFFFFull, chrom);
        const uint32_t k = (uint32_t)(sm_draw(sm_key(m.seed + file, file, 0xFFFFu), chrom) % m.num_hotspots);
        start = mul_hi(sm_draw(spots, k), chrom_len - 1000000u) + mul_hi(u2, 1000000u - len);
    } else {
        start = mul_hi(u2, chrom_len - len);
    }
    *s = start;
    *e = start + len;
}

Model model_of(uint64_t seed, double broad_fraction, double hotspot_fraction, uint32_t num_hotspots,
               uint32_t sid_base) {
    const double two53 = 9007199254740992.0;
    Model m;
    m.seed = seed;
    m.broad_thr = (uint64_t)(std::min(1.0, std::max(0.0, broad_fraction)) * two53);
    m.hot_thr = (uint64_t)(std::min(1.0, std::max(0.0, hotspot_fraction)) * two53);
    m.num_hotspots = num_hotspots;
    m.sid_base = sid_base;
    return m;
}

// Share of n intervals per chromosome: proportional to length, remainders by largest remainder
// (ties to the lower chromosome index).
void split_by_length(const uint32_t* chrom_len, uint32_t nc, uint64_t n, uint64_t* out) {
    unsigned __int128 total = 0;
    for (uint32_t c = 0; c < nc; c++) total += chrom_len[c];
    std::vector<std::pair<uint64_t, uint32_t>> rem;
    uint64_t given = 0;
    for (uint32_t c = 0; c < nc; c++) {
        const unsigned __int128 x = (unsigned __int128)n * chrom_len[c];
        out[c] = (uint64_t)(x / total);
        given += out[c];
        rem.push_back({(uint64_t)(x % total), c});
    }
    std::stable_sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    for (uint64_t k = 0; given < n; k++, given++) out[rem[k % nc].second]++;
}

uint32_t size_class(uint32_t min_size, uint32_t gf, uint32_t size) {
    // LayerConfig::layer_for_size (src/io/meta.rs:33-58): the smallest K with size < min_size * gf^K
    uint64_t thr = min_size;
    uint32_t k = 0;
    while (thr <= size) {
        thr = thr > UINT64_MAX / gf ? UINT64_MAX : thr * gf;
        k++;
    }
    return k;
}

}  // namespace

extern "C" {

void orc_synth_chrom_lengths(uint64_t seed, uint32_t nc, uint32_t* out) {
    const uint64_t key = sm_key(seed, 0xC0C0C0C0ull, 0);
    for (uint32_t c = 0; c < nc; c++) out[c] = 50000000u + mul_hi(sm_draw(key, c), 200000000u);
}

// Rank sizes round(C r^-s) clamped to [lo, hi], with C found by bisection so that they sum to target.
void orc_synth_zipf_sizes(uint32_t nf, double s, uint64_t lo, uint64_t hi, uint64_t target, uint64_t* out) {
    auto fill = [&](double c, bool write) {
        uint64_t sum = 0;
        for (uint32_t r = 1; r <= nf; r++) {
            const double v = std::round(c * std::pow((double)r, -s));
            const uint64_t n = v < (double)lo ? lo : (v > (double)hi ? hi : (uint64_t)v);
            if (write) out[r - 1] = n;
            sum += n;
        }
        return sum;
    };
    double a = 0.0, b = 1e20;
    for (int it = 0; it < 200; it++) {
        const double m = 0.5 * (a + b);
        if (fill(m, false) < target) a = m; else b = m;
    }
    fill(b, true);
}

void orc_synth_loguniform_sizes(uint64_t seed, uint32_t nf, uint64_t lo, uint64_t hi, uint64_t* out) {
    const uint64_t key = sm_key(seed, 0x512E5ull, 1);
    const double ll = std::log((double)lo), lh = std::log((double)hi);
    for (uint32_t f = 0; f < nf; f++) {
        const double u = (double)(sm_draw(key, f) >> 11) / 9007199254740992.0;
        const uint64_t n = (uint64_t)std::llround(std::exp(ll + (lh - ll) * u));
        out[f] = std::min(hi, std::max(lo, n));
    }
}

// Intervals of one (file, chromosome), sorted by (start, end): returns their number, writes them as
// (start, end, sid) triples when out is not NULL.
uint64_t orc_synth_block(uint64_t seed, const uint32_t* chrom_len, uint32_t nc, const uint64_t* file_sizes,
                         uint32_t file, uint32_t chrom, double broad_fraction, double hotspot_fraction,
                         uint32_t num_hotspots, uint32_t sid_base, uint32_t* out) {
    std::vector<uint64_t> per(nc);
    split_by_length(chrom_len, nc, file_sizes[file], per.data());
    const uint64_t n = per[chrom];
    if (!out) return n;
    const Model m = model_of(seed, broad_fraction, hotspot_fraction, num_hotspots, sid_base);
    std::vector<std::pair<uint32_t, uint32_t>> v(n);
    for (uint64_t i = 0; i < n; i++) one_interval(m, file, chrom, chrom_len[chrom], i, &v[i].first, &v[i].second);
    std::stable_sort(v.begin(), v.end());
    for (uint64_t i = 0; i < n; i++) {
        out[3 * i] = v[i].first;
        out[3 * i + 1] = v[i].second;
        out[3 * i + 2] = sid_base + file;
    }
    return n;
}

// The database layers of one chromosome: every file's intervals bucketed by size class and sorted
// by start within a class (ties in file, then generation order).  Returns the interval count; with
// pos / sid given, writes the classes back to back (class K's count in layer_counts[K]).
uint64_t orc_synth_chrom_layers(uint64_t seed, const uint32_t* chrom_len, uint32_t nc, const uint64_t* file_sizes,
                                uint32_t nf, uint32_t chrom, double broad_fraction, uint32_t sid_base,
                                uint32_t min_size, uint32_t gf, uint64_t* layer_counts, uint32_t max_layers,
                                uint32_t* pos, uint32_t* sid) {
    std::vector<uint64_t> per(nc), first(nf + 1, 0);
    for (uint32_t f = 0; f < nf; f++) {
        split_by_length(chrom_len, nc, file_sizes[f], per.data());
        first[f + 1] = first[f] + per[chrom];
    }
    const uint64_t total = first[nf];
    if (!pos || !sid) return total;
    const Model m = model_of(seed, broad_fraction, 0.0, 0, sid_base);
    std::vector<uint64_t> key(total), val(total);
    for (uint32_t f = 0; f < nf; f++)
        for (uint64_t i = 0; i < first[f + 1] - first[f]; i++) {
            uint32_t s, e;
            one_interval(m, f, chrom, chrom_len[chrom], i, &s, &e);
            key[first[f] + i] = ((uint64_t)size_class(min_size, gf, e - s) << 32) | s;
            val[first[f] + i] = ((uint64_t)e << 32) | (sid_base + f);
        }
    std::vector<uint64_t> order(total);
    std::iota(order.begin(), order.end(), 0ull);
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return key[a] < key[b]; });
    std::fill(layer_counts, layer_counts + max_layers, 0ull);
    for (uint64_t j = 0; j < total; j++) {
        const uint64_t k = key[order[j]], v = val[order[j]];
        const uint32_t K = (uint32_t)(k >> 32);
        if (K < max_layers) layer_counts[K]++;
        pos[2 * j] = (uint32_t)k;
        pos[2 * j + 1] = (uint32_t)(v >> 32);
        sid[j] = (uint32_t)v;
    }
    return total;
}

}  // extern "C"
