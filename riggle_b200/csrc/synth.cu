// Seeded synthetic interval workloads, identical on the host and on the device.
//
// Streams: SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014; finaliser constants as published by Vigna) evaluated as a counter-based generator:
// draw i of stream k is mix64(k + (i+1) * golden).  Every interval of (file f, chromosome c) uses
// four draws; lengths are read from host-built 65537-point quantile tables with integer
// interpolation, starts come from a 32x32-bit multiply-high, so host and device produce the same
// bits.  Interval model (per file): chromosome counts proportional to chromosome length (largest
// remainder), length ~ LogNormal(ln 500, 1) clipped to [20, 100000] bp, or with probability
// `broad_fraction` ~ LogUniform[10k, 1M]; with probability `hotspot_fraction` the interval is
// placed inside one of `num_hotspots` 1 Mbp hot spots shared across files, else start ~
// U[0, len - length).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace rgl {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t draw(uint64_t key, uint64_t i) {
    return mix64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
}
__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t file, uint64_t chrom) {
    return mix64(mix64(seed * 0xD1B54A32D192ED03ull + file) ^ (chrom * 0x8CB92BA72F3D8DD7ull + 0x632BE59BD9B4E019ull));
}
__host__ __device__ __forceinline__ uint32_t quantile(const uint32_t* T, uint64_t u) {
    uint32_t idx = (uint32_t)(u >> 48);
    uint32_t frac = (uint32_t)((u >> 32) & 0xFFFFu);
    uint32_t a = T[idx], b = T[idx + 1];
    return a + (uint32_t)(((uint64_t)(b - a) * frac) >> 16);
}
__host__ __device__ __forceinline__ uint32_t mulhi32(uint64_t u, uint32_t range) {
    return (uint32_t)(((u >> 32) * (uint64_t)range) >> 32);
}

struct GenParams {
    uint64_t seed;
    uint64_t broad_thr;  // compare (u >> 11) < thr  (53-bit)
    uint64_t hot_thr;
    uint32_t num_hotspots;
    uint32_t sid_base;
};

// One interval of (file, chrom) number i.
__host__ __device__ __forceinline__ void gen_interval(const GenParams& g, const uint32_t* t_logn, const uint32_t* t_logu,
                                                      uint32_t file, uint32_t chrom, uint32_t chrom_len, uint64_t i,
                                                      uint32_t* s_out, uint32_t* e_out) {
    uint64_t key = stream_key(g.seed + file, file, chrom);
    uint64_t u0 = draw(key, 4 * i), u1 = draw(key, 4 * i + 1), u2 = draw(key, 4 * i + 2), u3 = draw(key, 4 * i + 3);
    bool broad = (u0 >> 11) < g.broad_thr;
    bool hot = !broad && g.num_hotspots > 0 && (u3 >> 11) < g.hot_thr;
    uint32_t len = quantile(broad ? t_logu : t_logn, u1);
    if (len >= chrom_len) len = chrom_len - 1;
    uint32_t start;
    if (hot && chrom_len > 2000000u) {
        // hot-spot pool shared by all files: spot k of chromosome c
        uint64_t hk = stream_key(g.seed ^ 0x5151515151515151ull, 0xFFFFFFFFull, chrom);
        uint32_t k = (uint32_t)(draw(stream_key(g.seed + file, file, 0xFFFFu), chrom) % g.num_hotspots);
        uint32_t spot = mulhi32(draw(hk, k), chrom_len - 1000000u);
        start = spot + mulhi32(u2, 1000000u - len);
    } else {
        start = mulhi32(u2, chrom_len - len);
    }
    *s_out = start;
    *e_out = start + len;
}

// ---- host tables ---------------------------------------------------------------------------------
static double inv_norm(double p) {
    // Acklam's rational approximation of the standard normal quantile, refined by one Halley step
    // on erfc (P. J. Acklam, "An algorithm for computing the inverse normal cumulative
    // distribution function", 2003).
    static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                               1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                               6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                               -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                               3.754408661907416e+00};
    double q, r, x;
    if (p < 0.02425) {
        q = std::sqrt(-2 * std::log(p));
        x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
    } else if (p <= 1 - 0.02425) {
        q = p - 0.5;
        r = q * q;
        x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
    } else {
        q = std::sqrt(-2 * std::log(1 - p));
        x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
    }
    double e = 0.5 * std::erfc(-x / std::sqrt(2.0)) - p;
    double u = e * std::sqrt(2 * M_PI) * std::exp(x * x / 2);
    return x - u / (1 + x * u / 2);
}

const SynthTables& synth_tables() {
    static SynthTables t = [] {
        SynthTables s;
        s.lognormal.resize(65537);
        s.loguniform.resize(65537);
        for (int k = 0; k <= 65536; k++) {
            double v;
            if (k == 0) v = 20.0;
            else if (k == 65536) v = 100000.0;
            else v = std::exp(std::log(500.0) + 1.0 * inv_norm(k / 65536.0));
            v = std::min(100000.0, std::max(20.0, v));
            s.lognormal[k] = (uint32_t)std::llround(v);
            double w = 10000.0 * std::pow(100.0, k / 65536.0);
            s.loguniform[k] = (uint32_t)std::llround(std::min(1000000.0, w));
        }
        return s;
    }();
    return t;
}

static GenParams make_params(const rgl_synth_spec* sp) {
    GenParams g;
    g.seed = sp->seed;
    double bf = std::min(1.0, std::max(0.0, sp->broad_fraction));
    double hf = std::min(1.0, std::max(0.0, sp->hotspot_fraction));
    g.broad_thr = (uint64_t)(bf * 9007199254740992.0);
    g.hot_thr = (uint64_t)(hf * 9007199254740992.0);
    g.num_hotspots = sp->num_hotspots;
    g.sid_base = sp->sid_base;
    return g;
}

static void chrom_split(const rgl_synth_spec* sp, uint64_t n, uint64_t* out) {
    // proportional split of n over chromosome lengths, largest remainder (ties: lower index)
    unsigned __int128 L = 0;
    for (uint32_t c = 0; c < sp->num_chroms; c++) L += sp->chrom_len[c];
    uint64_t given = 0;
    std::vector<std::pair<uint64_t, uint32_t>> rem(sp->num_chroms);
    for (uint32_t c = 0; c < sp->num_chroms; c++) {
        unsigned __int128 x = (unsigned __int128)n * sp->chrom_len[c];
        out[c] = (uint64_t)(x / L);
        rem[c] = {(uint64_t)(x % L), c};
        given += out[c];
    }
    std::stable_sort(rem.begin(), rem.end(), [](auto& a, auto& b) { return a.first > b.first; });
    for (uint64_t k = 0; given < n; k++, given++) out[rem[k % sp->num_chroms].second]++;
}

static int check_spec(const rgl_synth_spec* sp) {
    if (!sp || !sp->chrom_len || !sp->file_sizes || sp->num_chroms == 0)
        return fail(RGL_ERR_INVALID_ARGUMENT, "incomplete synthetic spec");
    for (uint32_t c = 0; c < sp->num_chroms; c++)
        if (sp->chrom_len[c] < 1000) return fail(RGL_ERR_INVALID_ARGUMENT, "chromosome shorter than 1000 bp");
    return RGL_OK;
}

// ---- device generation of one chromosome --------------------------------------------------------
__global__ void k_synth_chrom(GenParams g, const uint32_t* __restrict__ t_logn, const uint32_t* __restrict__ t_logu,
                              uint32_t chrom, uint32_t chrom_len, const uint64_t* __restrict__ file_off,
                              uint32_t nfiles, uint32_t file_base, uint64_t total, uint32_t min_size, uint32_t gf,
                              uint64_t* __restrict__ key, uint64_t* __restrict__ val,
                              unsigned long long* __restrict__ layer_count, int count_only) {
    uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= total) return;
    uint32_t lo = 0, hi = nfiles;
    while (hi - lo > 1) {
        uint32_t m = (lo + hi) >> 1;
        if (file_off[m] <= j) lo = m; else hi = m;
    }
    uint32_t s, e;
    gen_interval(g, t_logn, t_logu, file_base + lo, chrom, chrom_len, j - file_off[lo], &s, &e);
    // layer_for_size (src/io/meta.rs:33-58), power-of-two path or threshold loop
    uint32_t size = e - s, K;
    if (size < min_size) K = 0;
    else if ((min_size & (min_size - 1)) == 0 && (gf & (gf - 1)) == 0 && gf >= 2) {
        uint32_t ls = 31u - __clz(size), lm = 31u - __clz(min_size), lg = __ffs(gf) - 1;
        K = (ls >= lm ? ls - lm : 0) / lg + 1;
    } else {
        uint64_t thr = min_size;
        K = 0;
        while (thr <= size) { thr = thr > 0xFFFFFFFFFFFFFFFFull / gf ? 0xFFFFFFFFFFFFFFFFull : thr * gf; K++; }
    }
    if (count_only) {
        atomicAdd(&layer_count[K], 1ull);
        return;
    }
    key[j] = ((uint64_t)K << 32) | s;
    val[j] = ((uint64_t)e << 32) | (g.sid_base + lo);
}

__global__ void k_synth_unpack(uint64_t total, const uint64_t* __restrict__ key, const uint64_t* __restrict__ val,
                               const uint64_t* __restrict__ kbegin, const uint64_t* __restrict__ koff,
                               uint32_t nslots, uint2* __restrict__ pos, uint32_t* __restrict__ sid) {
    uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= total) return;
    uint64_t k = key[j], v = val[j];
    uint32_t K = (uint32_t)(k >> 32);
    if (K >= nslots) return;
    uint64_t dst = koff[K] + (j - kbegin[K]);
    pos[dst] = make_uint2((uint32_t)k, (uint32_t)(v >> 32));
    sid[dst] = (uint32_t)v;
}

// One thread per interval of a file-major query batch: block b = (file b / C, chromosome b % C).
__global__ void k_synth_batch(GenParams g, const uint32_t* __restrict__ t_logn, const uint32_t* __restrict__ t_logu,
                              const uint32_t* __restrict__ chrom_len, uint32_t C, const uint64_t* __restrict__ off,
                              uint32_t nblk, uint64_t total, rgl_interval* __restrict__ out) {
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (j >= total) return;
    uint32_t lo = 0, hi = nblk;  // last block with off[b] <= j
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (off[m] <= j) lo = m; else hi = m;
    }
    const uint32_t f = lo / C, c = lo % C;
    uint32_t s, e;
    gen_interval(g, t_logn, t_logu, f, c, chrom_len[c], j - off[lo], &s, &e);
    out[j] = rgl_interval{s, e, g.sid_base + f};
}

}  // namespace rgl

using namespace rgl;

extern "C" {

int rgl_synth_chrom_lengths(uint64_t seed, uint32_t num_chroms, uint32_t* out) {
    if (!out) return fail(RGL_ERR_INVALID_ARGUMENT, "null output");
    uint64_t key = stream_key(seed, 0xC0C0C0C0ull, 0);
    for (uint32_t c = 0; c < num_chroms; c++) out[c] = 50000000u + mulhi32(draw(key, c), 200000000u);
    return RGL_OK;
}

int rgl_synth_zipf_sizes(uint32_t num_files, double s, uint64_t lo, uint64_t hi, uint64_t target, uint64_t* out) {
    if (!out || num_files == 0 || lo > hi) return fail(RGL_ERR_INVALID_ARGUMENT, "bad Zipf size arguments");
    auto total = [&](double C, bool write) {
        uint64_t sum = 0;
        for (uint32_t r = 1; r <= num_files; r++) {
            double v = std::round(C * std::pow((double)r, -s));
            uint64_t n = v < (double)lo ? lo : (v > (double)hi ? hi : (uint64_t)v);
            if (write) out[r - 1] = n;
            sum += n;
        }
        return sum;
    };
    double a = 0.0, b = 1e20;
    for (int it = 0; it < 200; it++) {
        double m = 0.5 * (a + b);
        if (total(m, false) < target) a = m; else b = m;
    }
    total(b, true);
    return RGL_OK;
}

int rgl_synth_loguniform_sizes(uint64_t seed, uint32_t num_files, uint64_t lo, uint64_t hi, uint64_t* out) {
    if (!out || lo == 0 || lo > hi) return fail(RGL_ERR_INVALID_ARGUMENT, "bad log-uniform size arguments");
    uint64_t key = stream_key(seed, 0x512E5ull, 1);
    double ll = std::log((double)lo), lh = std::log((double)hi);
    for (uint32_t f = 0; f < num_files; f++) {
        double u = (double)(draw(key, f) >> 11) / 9007199254740992.0;
        double v = std::exp(ll + (lh - ll) * u);
        uint64_t n = (uint64_t)std::llround(v);
        out[f] = std::min(hi, std::max(lo, n));
    }
    return RGL_OK;
}

int rgl_synth_file_chrom_counts(const rgl_synth_spec* sp, uint32_t file, uint64_t* out) {
    RGL_TRY(check_spec(sp));
    if (file >= sp->num_files || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "file index out of range");
    chrom_split(sp, sp->file_sizes[file], out);
    return RGL_OK;
}

int rgl_synth_block_host(const rgl_synth_spec* sp, uint32_t file, uint32_t chrom, rgl_interval* out, uint64_t capacity,
                         uint64_t* out_count) {
    RGL_TRY(check_spec(sp));
    if (file >= sp->num_files || chrom >= sp->num_chroms || !out_count)
        return fail(RGL_ERR_INVALID_ARGUMENT, "file/chrom out of range");
    std::vector<uint64_t> per(sp->num_chroms);
    chrom_split(sp, sp->file_sizes[file], per.data());
    uint64_t n = per[chrom];
    *out_count = n;
    if (!out) return RGL_OK;
    if (capacity < n) return fail(RGL_ERR_INVALID_ARGUMENT, "output capacity too small");
    const SynthTables& T = synth_tables();
    GenParams g = make_params(sp);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t s, e;
        gen_interval(g, T.lognormal.data(), T.loguniform.data(), file, chrom, sp->chrom_len[chrom], i, &s, &e);
        out[i] = rgl_interval{s, e, sp->sid_base + file};
    }
    std::stable_sort(out, out + n, [](const rgl_interval& a, const rgl_interval& b) {
        return a.start != b.start ? a.start < b.start : a.end < b.end;
    });
    return RGL_OK;
}

int rgl_synth_chrom_layers_host(const rgl_synth_spec* sp, uint32_t chrom, uint32_t min_size, uint32_t gf,
                                uint64_t* layer_counts, uint32_t max_layers, uint32_t* pos, uint32_t* sid,
                                uint64_t capacity, uint64_t* out_total) {
    RGL_TRY(check_spec(sp));
    if (chrom >= sp->num_chroms || !out_total || !layer_counts)
        return fail(RGL_ERR_INVALID_ARGUMENT, "bad chrom or null output");
    if (min_size == 0 || gf < 2) return fail(RGL_ERR_INVALID_ARGUMENT, "layer_config needs min_size >= 1, growth_factor >= 2");
    std::vector<uint64_t> per(sp->num_chroms);
    uint64_t total = 0;
    std::vector<uint64_t> foff(sp->num_files + 1, 0);
    for (uint32_t f = 0; f < sp->num_files; f++) {
        chrom_split(sp, sp->file_sizes[f], per.data());
        foff[f + 1] = foff[f] + per[chrom];
    }
    total = foff[sp->num_files];
    *out_total = total;
    if (!pos || !sid) return RGL_OK;
    if (capacity < total) return fail(RGL_ERR_INVALID_ARGUMENT, "output capacity too small");
    const SynthTables& T = synth_tables();
    GenParams g = make_params(sp);
    std::vector<uint64_t> key(total), val(total);
    for (uint32_t f = 0; f < sp->num_files; f++)
        for (uint64_t i = 0; i < foff[f + 1] - foff[f]; i++) {
            uint32_t s, e;
            gen_interval(g, T.lognormal.data(), T.loguniform.data(), f, chrom, sp->chrom_len[chrom], i, &s, &e);
            uint64_t K = layer_for_size(min_size, gf, e - s);
            key[foff[f] + i] = (K << 32) | s;
            val[foff[f] + i] = ((uint64_t)e << 32) | (sp->sid_base + f);
        }
    std::vector<uint64_t> order(total);
    for (uint64_t i = 0; i < total; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return key[a] < key[b]; });
    for (uint32_t K = 0; K < max_layers; K++) layer_counts[K] = 0;
    for (uint64_t j = 0; j < total; j++) {
        uint64_t k = key[order[j]], v = val[order[j]];
        uint32_t K = (uint32_t)(k >> 32);
        if (K < max_layers) layer_counts[K]++;
        pos[2 * j] = (uint32_t)k;
        pos[2 * j + 1] = (uint32_t)(v >> 32);
        sid[j] = (uint32_t)v;
    }
    return RGL_OK;
}

int rgl_synth_batch_layout(const rgl_synth_spec* sp, uint64_t* block_offsets, uint32_t* block_shards,
                           uint32_t* block_rows) {
    RGL_TRY(check_spec(sp));
    if (!block_offsets) return fail(RGL_ERR_INVALID_ARGUMENT, "null output");
    const uint32_t C = sp->num_chroms;
    std::vector<uint64_t> per(C);
    uint64_t acc = 0;
    for (uint32_t f = 0; f < sp->num_files; f++) {
        chrom_split(sp, sp->file_sizes[f], per.data());
        for (uint32_t c = 0; c < C; c++) {
            const uint64_t b = (uint64_t)f * C + c;
            block_offsets[b] = acc;
            if (block_shards) block_shards[b] = c;
            if (block_rows) block_rows[b] = f;
            acc += per[c];
        }
    }
    block_offsets[(uint64_t)sp->num_files * C] = acc;
    return RGL_OK;
}

int rgl_synth_batch_device(const rgl_synth_spec* sp, int device, const uint64_t* block_offsets, rgl_interval* d_out,
                           void* stream) {
    clear_error();
    RGL_TRY(check_spec(sp));
    if (!block_offsets) return fail(RGL_ERR_INVALID_ARGUMENT, "null block offsets");
    const uint64_t nblk = (uint64_t)sp->num_files * sp->num_chroms;
    const uint64_t total = block_offsets[nblk];
    if (total && !d_out) return fail(RGL_ERR_INVALID_ARGUMENT, "null output");
    if (nblk >= (1ull << 32)) return fail(RGL_ERR_INVALID_ARGUMENT, "too many blocks");
    RGL_CUDA(cudaSetDevice(device));
    if (!total) return RGL_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const SynthTables& T = synth_tables();
    DevBuf tn, tu, cl, off;
    int s = tn.ensure(65537 * 4);
    if (s == RGL_OK) s = tu.ensure(65537 * 4);
    if (s == RGL_OK) s = cl.ensure(sp->num_chroms * 4ull);
    if (s == RGL_OK) s = off.ensure((nblk + 1) * 8);
    if (s == RGL_OK &&
        (cudaMemcpy(tn.p, T.lognormal.data(), 65537 * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(tu.p, T.loguniform.data(), 65537 * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(cl.p, sp->chrom_len, sp->num_chroms * 4ull, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(off.p, block_offsets, (nblk + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess))
        s = fail(RGL_ERR_DEVICE, "synth upload");
    if (s == RGL_OK) {
        k_synth_batch<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
            make_params(sp), tn.as<uint32_t>(), tu.as<uint32_t>(), cl.as<uint32_t>(), sp->num_chroms,
            off.as<uint64_t>(), (uint32_t)nblk + 1, total, d_out);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "synth batch kernel");
    }
    for (DevBuf* b : {&tn, &tu, &cl, &off}) b->release();
    return s;
}

int rgl_index_synth(const rgl_synth_spec* sp, uint32_t min_size, uint32_t gf, int device, rgl_index** out) {
    return rgl_index_synth_columns(sp, min_size, gf, 0, sp ? sp->num_files : 0, device, out);
}

int rgl_index_synth_columns(const rgl_synth_spec* sp, uint32_t min_size, uint32_t gf, uint32_t file_lo,
                            uint32_t file_hi, int device, rgl_index** out) {
    clear_error();
    RGL_TRY(check_spec(sp));
    if (!out) return fail(RGL_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    if (min_size == 0 || gf < 2) return fail(RGL_ERR_INVALID_ARGUMENT, "layer_config needs min_size >= 1, growth_factor >= 2");
    if (file_lo > file_hi || file_hi > sp->num_files) return fail(RGL_ERR_INVALID_ARGUMENT, "bad file range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(RGL_ERR_NO_DEVICE, "no CUDA device");
    RGL_CUDA(cudaSetDevice(device));
    // files [file_lo, file_hi) keep their global streams; their sids are sid_base + (f - file_lo)
    const uint32_t C = sp->num_chroms, F = file_hi - file_lo;
    const uint32_t KMAX = 64;
    // per (file, chrom) counts and per-chromosome file offsets
    std::vector<uint64_t> fc((size_t)F * C);
    for (uint32_t f = 0; f < F; f++) chrom_split(sp, sp->file_sizes[file_lo + f], &fc[(size_t)f * C]);
    std::vector<std::vector<uint64_t>> foff(C, std::vector<uint64_t>(F + 1, 0));
    for (uint32_t c = 0; c < C; c++)
        for (uint32_t f = 0; f < F; f++) foff[c][f + 1] = foff[c][f] + fc[(size_t)f * C + c];
    for (uint32_t c = 0; c < C; c++)
        if (foff[c][F] >= (1ull << 31)) return fail(RGL_ERR_INVALID_ARGUMENT, "more than 2^31 intervals on one chromosome");

    const SynthTables& T = synth_tables();
    GenParams g = make_params(sp);
    uint32_t *d_tn = nullptr, *d_tu = nullptr;
    uint64_t* d_foff = nullptr;
    unsigned long long* d_cnt = nullptr;
    RGL_CUDA(cudaMalloc(&d_tn, 65537 * 4));
    RGL_CUDA(cudaMalloc(&d_tu, 65537 * 4));
    RGL_CUDA(cudaMalloc(&d_foff, (F + 1) * 8ull));
    RGL_CUDA(cudaMalloc(&d_cnt, (size_t)C * KMAX * 8));
    RGL_CUDA(cudaMemcpy(d_tn, T.lognormal.data(), 65537 * 4, cudaMemcpyHostToDevice));
    RGL_CUDA(cudaMemcpy(d_tu, T.loguniform.data(), 65537 * 4, cudaMemcpyHostToDevice));
    RGL_CUDA(cudaMemset(d_cnt, 0, (size_t)C * KMAX * 8));
    // pass A: per (chrom, layer) counts
    for (uint32_t c = 0; c < C; c++) {
        uint64_t tot = foff[c][F];
        if (!tot) continue;
        RGL_CUDA(cudaMemcpy(d_foff, foff[c].data(), (F + 1) * 8ull, cudaMemcpyHostToDevice));
        k_synth_chrom<<<(unsigned)((tot + 255) / 256), 256>>>(g, d_tn, d_tu, c, sp->chrom_len[c], d_foff, F, file_lo,
                                                              tot, min_size, gf, nullptr, nullptr,
                                                              d_cnt + (size_t)c * KMAX, 1);
    }
    RGL_CUDA(cudaGetLastError());
    std::vector<unsigned long long> cnt((size_t)C * KMAX);
    RGL_CUDA(cudaMemcpy(cnt.data(), d_cnt, cnt.size() * 8, cudaMemcpyDeviceToHost));

    auto* idx = new rgl_index();
    idx->device = device;
    idx->min_size = min_size;
    idx->gf = gf;
    idx->num_sources = sp->sid_base + F;
    idx->num_shards = C;
    static const char* names24[] = {"chr1",  "chr2",  "chr3",  "chr4",  "chr5",  "chr6",  "chr7",  "chr8",
                                    "chr9",  "chr10", "chr11", "chr12", "chr13", "chr14", "chr15", "chr16",
                                    "chr17", "chr18", "chr19", "chr20", "chr21", "chr22", "chrX",  "chrY"};
    for (uint32_t c = 0; c < C; c++) {
        std::string nm = (C <= 24) ? names24[c] : "chr" + std::to_string(c + 1);
        idx->shard_names.push_back(nm);
        idx->shard_ids[nm] = c;
    }
    for (uint32_t d = 0; d < idx->num_sources; d++)
        idx->source_names.push_back("source_" + std::to_string(d + file_lo) + ".bed");  // the global name
    for (uint32_t c = 0; c < C; c++)
        for (uint32_t K = 0; K < KMAX; K++)
            if (cnt[(size_t)c * KMAX + K]) {
                LayerDev l{};
                l.n = cnt[(size_t)c * KMAX + K];
                l.shard = c;
                l.layer = K;
                l.max_size = layer_max_size(min_size, gf, K);
                idx->layers.push_back(l);
                idx->total += l.n;
            }
    uint32_t maxk = 0;
    for (auto& l : idx->layers) maxk = std::max(maxk, l.layer + 1);
    idx->num_slots = maxk;
    idx->slot.assign((size_t)C * maxk, -1);
    for (size_t i = 0; i < idx->layers.size(); i++)
        idx->slot[(size_t)idx->layers[i].shard * maxk + idx->layers[i].layer] = (int32_t)i;
    int s = index_alloc(idx);
    // pass B: per chromosome generate, sort by (layer, start), scatter into the layer blocks
    uint64_t maxtot = 0;
    for (uint32_t c = 0; c < C; c++) maxtot = std::max(maxtot, foff[c][F]);
    DevBuf ka, kb, va, vb, tmp, kbeg, koff;
    if (s == RGL_OK) s = ka.ensure(maxtot * 8 + 8);
    if (s == RGL_OK) s = kb.ensure(maxtot * 8 + 8);
    if (s == RGL_OK) s = va.ensure(maxtot * 8 + 8);
    if (s == RGL_OK) s = vb.ensure(maxtot * 8 + 8);
    if (s == RGL_OK) s = kbeg.ensure(KMAX * 8);
    if (s == RGL_OK) s = koff.ensure(KMAX * 8);
    size_t tb = 0;
    int kbits = 1;
    while ((1u << kbits) < std::max<uint32_t>(maxk, 2)) kbits++;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint64_t*)nullptr, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (uint64_t*)nullptr, (int)std::max<uint64_t>(maxtot, 1), 0, 32 + kbits);
    if (s == RGL_OK) s = tmp.ensure(tb + 256);
    for (uint32_t c = 0; c < C && s == RGL_OK; c++) {
        uint64_t tot = foff[c][F];
        if (!tot) continue;
        std::vector<uint64_t> hb(KMAX, 0), ho(KMAX, 0);
        uint64_t acc = 0;
        for (uint32_t K = 0; K < maxk; K++) {
            hb[K] = acc;
            acc += cnt[(size_t)c * KMAX + K];
            int32_t li = idx->slot[(size_t)c * maxk + K];
            ho[K] = li >= 0 ? idx->layers[li].off : 0;
        }
        if (cudaMemcpy(d_foff, foff[c].data(), (F + 1) * 8ull, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(kbeg.p, hb.data(), KMAX * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(koff.p, ho.data(), KMAX * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
            s = fail(RGL_ERR_DEVICE, "synth upload");
            break;
        }
        k_synth_chrom<<<(unsigned)((tot + 255) / 256), 256>>>(g, d_tn, d_tu, c, sp->chrom_len[c], d_foff, F, file_lo,
                                                              tot, min_size, gf, ka.as<uint64_t>(), va.as<uint64_t>(),
                                                              nullptr, 0);
        size_t tbb = tmp.cap;
        if (cub::DeviceRadixSort::SortPairs(tmp.p, tbb, ka.as<uint64_t>(), kb.as<uint64_t>(), va.as<uint64_t>(),
                                            vb.as<uint64_t>(), (int)tot, 0, 32 + kbits) != cudaSuccess) {
            s = fail(RGL_ERR_DEVICE, "synth sort");
            break;
        }
        k_synth_unpack<<<(unsigned)((tot + 255) / 256), 256>>>(tot, kb.as<uint64_t>(), vb.as<uint64_t>(),
                                                               kbeg.as<uint64_t>(), koff.as<uint64_t>(), maxk,
                                                               idx->d_pos, idx->d_sid);
        if (cudaGetLastError() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "synth kernels");
    }
    if (s == RGL_OK && cudaDeviceSynchronize() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "synth sync");
    for (DevBuf* b : {&ka, &kb, &va, &vb, &tmp, &kbeg, &koff}) b->release();
    cudaFree(d_tn);
    cudaFree(d_tu);
    cudaFree(d_foff);
    cudaFree(d_cnt);
    if (s == RGL_OK) s = index_finalize(idx);
    if (s != RGL_OK) {
        index_free(idx);
        delete idx;
        return s;
    }
    *out = idx;
    return RGL_OK;
}

}  // extern "C"
