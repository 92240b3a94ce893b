// Host-side pieces of libriggle_b200: status strings, the thread-local error detail, the layer
// configuration arithmetic (src/io/meta.rs:33-81) and the meta.json reader (src/io/meta.rs:124-127).
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>

#include "internal.h"

namespace rgl {

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
void clear_error() {
    g_last_error.clear();
    (void)cudaGetLastError();  // a failed call of an earlier, unrelated operation must not leak into this one
}

static inline bool is_pow2(uint32_t x) { return x != 0 && (x & (x - 1)) == 0; }

uint32_t layer_for_size(uint32_t min_size, uint32_t gf, uint32_t size) {
    // Power-of-two fast path and the general threshold loop of src/io/meta.rs:33-58.  The caller
    // has validated min_size >= 1 and growth_factor >= 2 (the reference's loop never ends otherwise).
    if (size < min_size) return 0;
    if (is_pow2(min_size) && is_pow2(gf) && gf >= 2) {
        uint32_t ls = 31u - (uint32_t)__builtin_clz(size);
        uint32_t lm = 31u - (uint32_t)__builtin_clz(min_size);
        uint32_t lg = (uint32_t)__builtin_ctz(gf);
        return (ls >= lm ? ls - lm : 0) / lg + 1;
    }
    if (min_size == 0 || gf < 2) return 0;
    uint64_t thr = min_size;
    uint32_t k = 0;
    while (thr <= size) {
        unsigned __int128 t = (unsigned __int128)thr * gf;
        thr = t > UINT64_MAX ? UINT64_MAX : (uint64_t)t;
        k++;
    }
    return k;
}

uint32_t layer_max_size(uint32_t min_size, uint32_t gf, uint32_t layer) {
    uint64_t v = min_size;
    for (uint32_t i = 0; i < layer; i++) {
        unsigned __int128 t = (unsigned __int128)v * gf;
        v = t > UINT64_MAX ? UINT64_MAX : (uint64_t)t;
    }
    return v > UINT32_MAX ? UINT32_MAX : (uint32_t)v;
}

uint32_t tile_size(uint32_t min_size, uint32_t gf, uint32_t layer) {
    uint32_t t = layer_max_size(min_size, gf, layer) / 2;
    return t < 1 ? 1 : t;
}

bool file_exists(const std::string& path) {
    struct stat st;
    return ::stat(path.c_str(), &st) == 0;
}

int read_file(const std::string& path, std::vector<uint8_t>* out) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(RGL_ERR_IO, "cannot open " + path + ": " + std::strerror(errno));
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out->resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? std::fread(out->data(), 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if ((long)got != sz) return fail(RGL_ERR_IO, "short read of " + path);
    return RGL_OK;
}

// ---- minimal JSON reader for meta.json ---------------------------------------------------------
namespace {
struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    double num = 0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;
    const JVal* get(const char* k) const {
        for (auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct JParser {
    const char* p;
    const char* e;
    std::string err;
    void ws() {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
    }
    bool lit(const char* s) {
        size_t n = std::strlen(s);
        if ((size_t)(e - p) >= n && std::memcmp(p, s, n) == 0) {
            p += n;
            return true;
        }
        return false;
    }
    bool str(std::string* out) {
        if (p >= e || *p != '"') return false;
        p++;
        while (p < e && *p != '"') {
            if (*p == '\\') {
                p++;
                if (p >= e) return false;
                char c = *p++;
                switch (c) {
                    case 'n': out->push_back('\n'); break;
                    case 't': out->push_back('\t'); break;
                    case 'r': out->push_back('\r'); break;
                    case 'b': out->push_back('\b'); break;
                    case 'f': out->push_back('\f'); break;
                    case 'u': {
                        if (e - p < 4) return false;
                        unsigned cp = (unsigned)std::strtoul(std::string(p, p + 4).c_str(), nullptr, 16);
                        p += 4;
                        if (cp < 0x80) out->push_back((char)cp);
                        else if (cp < 0x800) {
                            out->push_back((char)(0xC0 | (cp >> 6)));
                            out->push_back((char)(0x80 | (cp & 0x3F)));
                        } else {
                            out->push_back((char)(0xE0 | (cp >> 12)));
                            out->push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
                            out->push_back((char)(0x80 | (cp & 0x3F)));
                        }
                        break;
                    }
                    default: out->push_back(c);
                }
            } else
                out->push_back(*p++);
        }
        if (p >= e) return false;
        p++;
        return true;
    }
    bool val(JVal* v, int depth) {
        if (depth > 64) return false;
        ws();
        if (p >= e) return false;
        if (*p == '{') {
            p++;
            v->kind = JVal::OBJ;
            ws();
            if (p < e && *p == '}') { p++; return true; }
            for (;;) {
                ws();
                std::string k;
                if (!str(&k)) return false;
                ws();
                if (p >= e || *p != ':') return false;
                p++;
                JVal c;
                if (!val(&c, depth + 1)) return false;
                v->obj.emplace_back(std::move(k), std::move(c));
                ws();
                if (p < e && *p == ',') { p++; continue; }
                if (p < e && *p == '}') { p++; return true; }
                return false;
            }
        }
        if (*p == '[') {
            p++;
            v->kind = JVal::ARR;
            ws();
            if (p < e && *p == ']') { p++; return true; }
            for (;;) {
                JVal c;
                if (!val(&c, depth + 1)) return false;
                v->arr.push_back(std::move(c));
                ws();
                if (p < e && *p == ',') { p++; continue; }
                if (p < e && *p == ']') { p++; return true; }
                return false;
            }
        }
        if (*p == '"') {
            v->kind = JVal::STR;
            return str(&v->str);
        }
        if (lit("true")) { v->kind = JVal::BOOL; v->num = 1; return true; }
        if (lit("false")) { v->kind = JVal::BOOL; v->num = 0; return true; }
        if (lit("null")) { v->kind = JVal::NUL; return true; }
        char* end = nullptr;
        std::string tmp(p, std::min<size_t>(64, (size_t)(e - p)));
        double d = std::strtod(tmp.c_str(), &end);
        if (end == tmp.c_str()) return false;
        p += (end - tmp.c_str());
        v->kind = JVal::NUM;
        v->num = d;
        return true;
    }
};
}  // namespace

int meta_load(const std::string& db_dir, MetaInfo* out) {
    // Meta::load (src/io/meta.rs:124-127): serde_json of {sid_map, layer_config, shards, num_layers}.
    std::vector<uint8_t> buf;
    RGL_TRY(read_file(db_dir + "/meta.json", &buf));
    JParser jp{reinterpret_cast<const char*>(buf.data()), reinterpret_cast<const char*>(buf.data()) + buf.size(), {}};
    JVal root;
    if (!jp.val(&root, 0) || root.kind != JVal::OBJ) return fail(RGL_ERR_META_JSON, "meta.json: malformed JSON");
    const JVal* sm = root.get("sid_map");
    const JVal* lc = root.get("layer_config");
    const JVal* sh = root.get("shards");
    const JVal* nl = root.get("num_layers");
    if (!sm || sm->kind != JVal::OBJ || !lc || lc->kind != JVal::OBJ || !sh || sh->kind != JVal::ARR || !nl ||
        nl->kind != JVal::NUM)
        return fail(RGL_ERR_META_JSON, "meta.json: missing field (sid_map, layer_config, shards, num_layers)");
    for (auto& kv : sm->obj) {
        char* end = nullptr;
        unsigned long sid = std::strtoul(kv.first.c_str(), &end, 10);
        if (end == kv.first.c_str() || *end != '\0' || sid > UINT32_MAX)
            return fail(RGL_ERR_META_JSON, "meta.json: sid_map key '" + kv.first + "' is not a u32");
        const JVal* name = kv.second.get("name");
        if (!name || name->kind != JVal::STR) return fail(RGL_ERR_META_JSON, "meta.json: sid_map entry without name");
        out->sid_map[(uint32_t)sid] = name->str;
    }
    const JVal* ms = lc->get("min_size");
    const JVal* g = lc->get("growth_factor");
    if (!ms || ms->kind != JVal::NUM || !g || g->kind != JVal::NUM)
        return fail(RGL_ERR_META_JSON, "meta.json: layer_config needs min_size and growth_factor");
    out->min_size = (uint32_t)ms->num;
    out->growth_factor = (uint32_t)g->num;
    for (auto& s : sh->arr) {
        if (s.kind != JVal::STR) return fail(RGL_ERR_META_JSON, "meta.json: shard name is not a string");
        out->shards.push_back(s.str);
    }
    out->num_layers = (uint64_t)nl->num;
    return RGL_OK;
}

}  // namespace rgl

// ================================================================================================
// C ABI: status, version, layer config
// ================================================================================================
extern "C" {

const char* rgl_status_str(int s) {
    switch (s) {
        case RGL_OK: return "ok";
        case RGL_ERR_INVALID_ARGUMENT: return "invalid argument";
        case RGL_ERR_IO: return "IO error";
        case RGL_ERR_BED_INVALID_FORMAT: return "BED parse error: invalid format - expected at least 2 integer columns";
        case RGL_ERR_BED_INVALID_START: return "BED parse error: invalid start coordinate";
        case RGL_ERR_BED_INVALID_END: return "BED parse error: invalid end coordinate";
        case RGL_ERR_BED_INVALID_RANGE: return "BED parse error: start must be less than end";
        case RGL_ERR_META_JSON: return "Meta error: JSON error";
        case RGL_ERR_LAYER_INVALID_POSITION_SIZE: return "Layer error: position file has invalid size";
        case RGL_ERR_LAYER_INVALID_SID_SIZE: return "Layer error: sid file has invalid size";
        case RGL_ERR_LAYER_SID_SIZE_MISMATCH: return "Layer error: position count does not match sid count";
        case RGL_ERR_LAYER_INVALID_INDEX_SIZE: return "Layer error: index file has invalid size";
        case RGL_ERR_DATABASE_NOT_FOUND: return "Database not found";
        case RGL_ERR_INPUT_NOT_FOUND: return "Input path not found";
        case RGL_ERR_NO_BED_FILES: return "No BED files found";
        case RGL_ERR_OOM: return "device out of memory";
        case RGL_ERR_TIMEOUT: return "device wait timed out";
        case RGL_ERR_DEVICE: return "CUDA error";
        case RGL_ERR_INDEX_INVARIANT: return "index invariant violated";
        case RGL_ERR_NO_DEVICE: return "no CUDA device";
        case RGL_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* rgl_last_error(void) { return rgl::g_last_error.c_str(); }
int rgl_version(void) { return 100; }

uint32_t rgl_layer_for_size(uint32_t min_size, uint32_t growth_factor, uint32_t size) {
    return rgl::layer_for_size(min_size, growth_factor, size);
}
uint32_t rgl_layer_max_size(uint32_t min_size, uint32_t growth_factor, uint32_t layer) {
    return rgl::layer_max_size(min_size, growth_factor, layer);
}
uint32_t rgl_tile_size(uint32_t min_size, uint32_t growth_factor, uint32_t layer) {
    return rgl::tile_size(min_size, growth_factor, layer);
}

}  // extern "C"
