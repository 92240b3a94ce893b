// BED ingest for the query path: parse_bed_line / parse_bed_file (src/io/parse.rs:47-141) and
// enumerate_query_files / parse_file_batch (src/tasks/query/files.rs:25-111), natively on the host.
//
// Line rules kept from the reference: the line is trimmed; empty lines and lines starting with '#'
// are skipped; whitespace-separated tokens are scanned left to right, the first two that parse as
// u32 (optional '+', decimal digits, at most 4294967295 — a longer number is not an integer and
// can become the shard name) are start and end, the first other token is the shard ("default"
// when none); scanning stops once a shard and an end are known.  Fewer than two tokens, or a
// missing start / end, is InvalidFormat; start >= end is InvalidRange; both carry the 1-based line
// number.  `.gz` files are read through zlib's gzread, which continues across concatenated gzip
// members as MultiGzDecoder does.  Whitespace is ASCII whitespace and bytes are not checked as
// UTF-8 (the reference trims and splits on Unicode whitespace and rejects invalid UTF-8 lines).
//
// A batch enumerates the *.bed / *.bed.gz files of a directory sorted by path (or takes one file),
// parses them on several threads, drops files with no intervals and numbers the remaining ones
// 0.. in path order (the compact Q_SIDs), keeping per file its shards in first-appearance order.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <dirent.h>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unordered_map>

#include "internal.h"

using rgl::BedFile;

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Rust's u32::from_str: an optional '+', then one or more decimal digits, no overflow.
bool parse_u32(const char* b, const char* e, uint32_t* out) {
    if (b < e && *b == '+') b++;
    if (b == e) return false;
    uint64_t v = 0;
    for (const char* p = b; p < e; p++) {
        if (*p < '0' || *p > '9') return false;
        v = v * 10 + (uint64_t)(*p - '0');
        if (v > 0xFFFFFFFFull) return false;
    }
    *out = (uint32_t)v;
    return true;
}

// One line; returns RGL_OK with *skip for comments and blank lines.
int parse_line(const char* b, const char* e, uint64_t line, uint32_t sid, BedFile* f,
               std::unordered_map<std::string, uint32_t>* index, bool* skip) {
    while (b < e && is_ws(*b)) b++;
    while (e > b && is_ws(e[-1])) e--;
    *skip = (b == e || *b == '#');
    if (*skip) return RGL_OK;
    const char *sb = nullptr, *se = nullptr;
    bool have_s = false, have_e = false;
    uint32_t start = 0, end = 0;
    int cols = 0;
    const char* p = b;
    while (p < e) {
        while (p < e && is_ws(*p)) p++;
        if (p == e) break;
        const char* t = p;
        while (p < e && !is_ws(*p)) p++;
        cols++;
        uint32_t v;
        if (parse_u32(t, p, &v)) {
            if (!have_s) { start = v; have_s = true; }
            else if (!have_e) { end = v; have_e = true; }
        } else if (!sb) {
            sb = t;
            se = p;
        }
        if (sb && have_e) break;
    }
    if (cols < 2 || !have_s || !have_e)
        return rgl::fail(RGL_ERR_BED_INVALID_FORMAT,
                         "Line " + std::to_string(line) + ": invalid format - expected at least 2 integer columns");
    if (start >= end)
        return rgl::fail(RGL_ERR_BED_INVALID_RANGE, "Line " + std::to_string(line) + ": start (" +
                                                        std::to_string(start) + ") must be less than end (" +
                                                        std::to_string(end) + ")");
    std::string shard = sb ? std::string(sb, se) : std::string("default");
    auto it = index->find(shard);
    uint32_t k;
    if (it == index->end()) {
        k = (uint32_t)f->shards.size();
        index->emplace(shard, k);
        f->shards.push_back(shard);
        f->ivs.emplace_back();
    } else {
        k = it->second;
    }
    f->ivs[k].push_back(rgl_interval{start, end, sid});
    f->count++;
    return RGL_OK;
}

int parse_buffer(const char* data, uint64_t len, uint32_t sid, BedFile* f) {
    std::unordered_map<std::string, uint32_t> index;
    uint64_t line = 0, at = 0;
    while (at < len) {
        const char* b = data + at;
        const char* nl = static_cast<const char*>(memchr(b, '\n', len - at));
        const char* e = nl ? nl : data + len;
        line++;
        bool skip;
        RGL_TRY(parse_line(b, e, line, sid, f, &index, &skip));
        at = (uint64_t)(e - data) + 1;
    }
    return RGL_OK;
}

bool ends_with(const std::string& s, const char* suf) {
    const size_t n = strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

}  // namespace

namespace rgl {

int bed_read(const std::string& path, uint32_t sid, BedFile* f) {
    std::vector<char> buf;
    if (ends_with(path, ".gz")) {
        gzFile g = gzopen(path.c_str(), "rb");
        if (!g) return rgl::fail(RGL_ERR_IO, "cannot open " + path);
        std::vector<char> chunk(1 << 20);
        for (;;) {
            const int r = gzread(g, chunk.data(), (unsigned)chunk.size());
            if (r < 0) {
                int en = 0;
                std::string msg = gzerror(g, &en);
                gzclose(g);
                return rgl::fail(RGL_ERR_IO, path + ": " + msg);
            }
            if (r == 0) break;
            buf.insert(buf.end(), chunk.data(), chunk.data() + r);
        }
        gzclose(g);
    } else {
        std::vector<uint8_t> raw;
        RGL_TRY(rgl::read_file(path, &raw));
        buf.assign(raw.begin(), raw.end());
    }
    const size_t slash = path.find_last_of('/');
    f->name = slash == std::string::npos ? path : path.substr(slash + 1);
    return parse_buffer(buf.data(), buf.size(), sid, f);
}

bool is_bed_name(const std::string& n) { return ends_with(n, ".bed") || ends_with(n, ".bed.gz"); }

int bed_list(const std::string& root, std::vector<std::string>* paths, bool* is_dir) {
    struct stat stt;
    if (stat(root.c_str(), &stt) != 0) return fail(RGL_ERR_INPUT_NOT_FOUND, "input path not found: " + root);
    *is_dir = S_ISDIR(stt.st_mode);
    if (*is_dir) {
        DIR* d = opendir(root.c_str());
        if (!d) return fail(RGL_ERR_IO, "cannot list " + root);
        while (dirent* e = readdir(d)) {
            std::string n = e->d_name;
            if (!is_bed_name(n)) continue;
            std::string p = root + (root.back() == '/' ? "" : "/") + n;
            struct stat fs;
            if (stat(p.c_str(), &fs) == 0 && S_ISREG(fs.st_mode)) paths->push_back(p);
        }
        closedir(d);
        std::sort(paths->begin(), paths->end());
    } else {
        paths->push_back(root);
    }
    return RGL_OK;
}

int bed_read_all(const std::vector<std::string>& paths, uint32_t sid0, uint32_t threads, std::vector<BedFile>* out) {
    out->assign(paths.size(), BedFile());
    std::vector<int> status(paths.size(), RGL_OK);
    std::vector<std::string> errs(paths.size());
    std::atomic<size_t> next{0};
    const uint32_t nt = std::max<uint32_t>(1, std::min<uint32_t>(threads ? threads : std::thread::hardware_concurrency(),
                                                                 (uint32_t)std::max<size_t>(paths.size(), 1)));
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < paths.size();) {
            status[i] = bed_read(paths[i], sid0 + (uint32_t)i, &(*out)[i]);
            if (status[i] != RGL_OK) errs[i] = rgl_last_error();
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (size_t i = 0; i < paths.size(); i++)  // the first failing file in path order
        if (status[i] != RGL_OK) return fail(status[i], paths[i] + ": " + errs[i]);
    return RGL_OK;
}

}  // namespace rgl

using namespace rgl;

struct rgl_bed_batch {
    std::vector<BedFile> files;  // non-empty files, row = position
};

extern "C" {

int rgl_bed_parse_string(const char* text, uint64_t len, uint32_t sid, rgl_bed_batch** out) {
    rgl::clear_error();
    if (!out || (!text && len)) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto* b = new rgl_bed_batch();
    BedFile f;
    f.name = "string";
    int s = parse_buffer(text, len, sid, &f);
    if (s != RGL_OK) {
        delete b;
        return s;
    }
    b->files.push_back(std::move(f));  // kept even when empty: a single parse result
    *out = b;
    return RGL_OK;
}

int rgl_bed_batch_load(const char* query_path, uint32_t threads, rgl_bed_batch** out) {
    rgl::clear_error();
    if (!query_path || !out) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::vector<std::string> paths;
    bool is_dir = false;
    RGL_TRY(bed_list(query_path, &paths, &is_dir));  // files.sort() (files.rs:33)
    std::vector<BedFile> parsed;
    RGL_TRY(bed_read_all(paths, 0, threads, &parsed));
    auto* b = new rgl_bed_batch();
    for (size_t i = 0; i < paths.size(); i++) {
        if (!parsed[i].count) continue;  // empty files get no Q_SID (files.rs:80-82)
        const uint32_t row = (uint32_t)b->files.size();
        for (auto& v : parsed[i].ivs)
            for (auto& iv : v) iv.sid = row;
        b->files.push_back(std::move(parsed[i]));
    }
    *out = b;
    return RGL_OK;
}

uint32_t rgl_bed_batch_rows(const rgl_bed_batch* b) { return b ? (uint32_t)b->files.size() : 0; }

const char* rgl_bed_batch_row_name(const rgl_bed_batch* b, uint32_t row) {
    return (b && row < b->files.size()) ? b->files[row].name.c_str() : nullptr;
}

uint64_t rgl_bed_batch_row_count(const rgl_bed_batch* b, uint32_t row) {
    return (b && row < b->files.size()) ? b->files[row].count : 0;
}

uint32_t rgl_bed_batch_row_shards(const rgl_bed_batch* b, uint32_t row) {
    return (b && row < b->files.size()) ? (uint32_t)b->files[row].shards.size() : 0;
}

int rgl_bed_batch_block(const rgl_bed_batch* b, uint32_t row, uint32_t k, const char** shard,
                        const rgl_interval** intervals, uint64_t* count) {
    if (!b || row >= b->files.size() || k >= b->files[row].shards.size())
        return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "no such block");
    if (shard) *shard = b->files[row].shards[k].c_str();
    if (intervals) *intervals = b->files[row].ivs[k].data();
    if (count) *count = b->files[row].ivs[k].size();
    return RGL_OK;
}

int rgl_bed_batch_query(rgl_context* ctx, const rgl_bed_batch* b, const rgl_query_opts* opts, uint32_t* counts,
                        uint64_t* overlap_bp, rgl_query_stats* stats) {
    rgl::clear_error();
    if (!ctx || !b || !counts) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<rgl_query_shard> shards;
    for (const BedFile& f : b->files)
        for (size_t k = 0; k < f.shards.size(); k++)
            shards.push_back(rgl_query_shard{f.shards[k].c_str(), 0, f.ivs[k].size(), f.ivs[k].data()});
    rgl_query_batch qb{(uint32_t)b->files.size(), (uint32_t)shards.size(), shards.data()};
    return rgl_query_counts(ctx, &qb, opts, counts, overlap_bp, stats);
}

int rgl_bed_batch_free(rgl_bed_batch* b) {
    delete b;
    return RGL_OK;
}

}  // extern "C"
