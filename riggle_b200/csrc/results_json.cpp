// The query results as the reference writes them: `chuckle query` serialises a StatsOutput (or, in
// --intervals mode, an IntervalsOutput) with serde_json::to_string_pretty (src/main.rs:131-204,
// src/stats/mod.rs:1-60).  The layout is kept byte for byte: two-space indentation, "key": value
// pairs in field order, optional fields left out when absent, non-finite floats as null, and each
// f64 as the shortest decimal that reads back to the same double, placed the way serde_json's
// float printer places it (plain decimal for decimal exponents -5 < e <= 16 with a ".0" on
// integers, otherwise d.ddde<exp>).
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace {

// Shortest round-trip digits (std::to_chars, C++17) laid out by the rules described above.
void put_f64(std::string& o, double v) {
    if (!std::isfinite(v)) {
        o += "null";
        return;
    }
    if (v == 0.0) {
        o += std::signbit(v) ? "-0.0" : "0.0";
        return;
    }
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific);
    std::string sci(buf, r.ptr);  // [-]d[.ddd]e(+|-)xx
    std::string digits;
    bool neg = false;
    size_t i = 0;
    if (sci[0] == '-') {
        neg = true;
        i = 1;
    }
    const size_t epos = sci.find('e');
    for (size_t k = i; k < epos; k++)
        if (sci[k] != '.') digits += sci[k];
    const int exp10 = std::atoi(sci.c_str() + epos + 1);  // v = d.ddd x 10^exp10
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    const int length = (int)digits.size();
    const int kk = exp10 + 1;  // 10^(kk-1) <= |v| < 10^kk
    const int k = kk - length;  // v = digits x 10^k
    if (neg) o += '-';
    if (0 <= k && kk <= 16) {  // integer: digits, zeros, ".0"
        o += digits;
        o.append((size_t)k, '0');
        o += ".0";
    } else if (0 < kk && kk <= 16) {  // point inside the digits
        o += digits.substr(0, (size_t)kk);
        o += '.';
        o += digits.substr((size_t)kk);
    } else if (-5 < kk && kk <= 0) {  // 0.000ddd
        o += "0.";
        o.append((size_t)(-kk), '0');
        o += digits;
    } else {  // d.ddde<exp>, or de<exp> for one digit
        o += digits[0];
        if (length > 1) {
            o += '.';
            o += digits.substr(1);
        }
        o += 'e';
        o += std::to_string(kk - 1);
    }
}

// A JSON string as serde_json writes it: ", \ and control characters escaped, other bytes as they are.
void put_str(std::string& o, const char* s) {
    static const char* hex = "0123456789abcdef";
    o += '"';
    for (const unsigned char* p = reinterpret_cast<const unsigned char*>(s ? s : ""); *p; p++) {
        const unsigned char c = *p;
        switch (c) {
            case '"': o += "\\\""; break;
            case '\\': o += "\\\\"; break;
            case '\n': o += "\\n"; break;
            case '\r': o += "\\r"; break;
            case '\t': o += "\\t"; break;
            case '\b': o += "\\b"; break;
            case '\f': o += "\\f"; break;
            default:
                if (c < 0x20) {
                    o += "\\u00";
                    o += hex[c >> 4];
                    o += hex[c & 15];
                } else {
                    o += (char)c;
                }
        }
    }
    o += '"';
}

void put_u64(std::string& o, uint64_t v) { o += std::to_string(v); }

struct Field {
    const char* key;
    int kind;  // 0 string, 1 integer, 2 f64
    const char* s;
    uint64_t u;
    double d;
};

void put_object(std::string& o, const std::vector<Field>& fs) {
    o += "    {\n";
    for (size_t i = 0; i < fs.size(); i++) {
        o += "      \"";
        o += fs[i].key;
        o += "\": ";
        if (fs[i].kind == 0) put_str(o, fs[i].s);
        else if (fs[i].kind == 1) put_u64(o, fs[i].u);
        else put_f64(o, fs[i].d);
        if (i + 1 < fs.size()) o += ',';
        o += '\n';
    }
    o += "    }";
}

int deliver(const std::string& o, char* out, uint64_t capacity, uint64_t* out_len) {
    *out_len = o.size();
    if (!out) return RGL_OK;
    if (capacity < o.size()) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "output capacity too small");
    std::memcpy(out, o.data(), o.size());
    return RGL_OK;
}

}  // namespace

extern "C" {

int rgl_format_stats_json(uint32_t num_rows, uint32_t num_sources, const char* const* query_names,
                          const char* const* db_names, const uint64_t* indptr, const uint32_t* indices,
                          const uint32_t* counts, const double* observed_bins, const double* p_value,
                          const double* llr, const uint8_t* flags, char* out, uint64_t capacity,
                          uint64_t* out_len) {
    rgl::clear_error();
    if (!out_len || !indptr || (indptr[num_rows] && (!indices || !counts)))
        return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    const bool stats = p_value != nullptr;
    if (stats && (!observed_bins || !flags))
        return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "stats output needs observed_bins, p_value and flags");
    struct Entry {
        uint32_t row, col, count;
        double obs, p, llr;
        bool has_llr;
    };
    std::vector<Entry> es;
    for (uint32_t q = 0; q < num_rows; q++) {
        if (indptr[q + 1] < indptr[q]) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "row pointers must not decrease");
        for (uint64_t e = indptr[q]; e < indptr[q + 1]; e++) {
            const uint32_t d = indices[e];
            if (d >= num_sources) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "column index >= num_sources");
            if (!stats) {
                es.push_back(Entry{q, d, counts[e], 0, 0, 0, false});
                continue;
            }
            const uint64_t cell = (uint64_t)q * num_sources + d;
            if (!(flags[cell] & RGL_PV_EMITTED)) continue;  // no shared chromosome: the reference emits nothing
            es.push_back(Entry{q, d, counts[e], observed_bins[cell], p_value[cell], llr ? llr[cell] : 0.0,
                               llr && (flags[cell] & RGL_PV_HAS_LLR)});
        }
    }
    // the reference's order: ascending p-value with stats (ties in (query, database) order here;
    // the reference's tie order follows a HashMap), descending overlap count without (stable over
    // the row-major CSR order, as the reference's)
    if (stats)
        std::stable_sort(es.begin(), es.end(), [](const Entry& a, const Entry& b) {
            if (std::isnan(a.p) || std::isnan(b.p)) return !std::isnan(a.p) && std::isnan(b.p);
            return a.p < b.p;
        });
    else
        std::stable_sort(es.begin(), es.end(), [](const Entry& a, const Entry& b) { return a.count > b.count; });
    std::string o = "{\n  \"results\": [";
    for (size_t i = 0; i < es.size(); i++) {
        const Entry& e = es[i];
        o += i ? ",\n" : "\n";
        std::vector<Field> fs = {{"query_name", 0, query_names ? query_names[e.row] : "", 0, 0},
                                 {"db_name", 0, db_names ? db_names[e.col] : "", 0, 0},
                                 {"overlap_count", 1, nullptr, e.count, 0}};
        if (stats) {
            fs.push_back({"observed_bins", 2, nullptr, 0, e.obs});
            fs.push_back({"p_value", 2, nullptr, 0, e.p});
            if (e.has_llr) fs.push_back({"llr", 2, nullptr, 0, e.llr});
        }
        put_object(o, fs);
    }
    o += es.empty() ? "]\n}" : "\n  ]\n}";
    return deliver(o, out, capacity, out_len);
}

int rgl_format_intervals_json(const rgl_pair* pairs, uint64_t n, uint32_t num_rows, uint32_t num_sources,
                              uint32_t num_shards, const char* const* query_names, const char* const* db_names,
                              const char* const* shard_names, char* out, uint64_t capacity, uint64_t* out_len) {
    rgl::clear_error();
    if (!out_len || (n && !pairs)) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    std::string o = "{\n  \"hits\": [";
    for (uint64_t i = 0; i < n; i++) {
        const rgl_pair& p = pairs[i];
        if (p.row >= num_rows || p.sid >= num_sources || p.shard >= num_shards)
            return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "pair row / sid / shard out of range");
        o += i ? ",\n" : "\n";
        put_object(o, {{"query_name", 0, query_names ? query_names[p.row] : "", 0, 0},
                       {"db_name", 0, db_names ? db_names[p.sid] : "", 0, 0},
                       {"chrom", 0, shard_names ? shard_names[p.shard] : "", 0, 0},
                       {"query_start", 1, nullptr, p.query_start, 0},
                       {"query_end", 1, nullptr, p.query_end, 0},
                       {"db_start", 1, nullptr, p.db_start, 0},
                       {"db_end", 1, nullptr, p.db_end, 0},
                       {"intersection_bp", 1, nullptr, p.intersection_bp, 0}});
    }
    o += n ? "\n  ]\n}" : "]\n}";
    return deliver(o, out, capacity, out_len);
}

}  // extern "C"
