// Index build on the device: add_to_database (src/tasks/build.rs:86-276) producing an HBM index,
// and the writer of the reference's on-disk layout.
//
// add: the database BED files (sorted by path; every file, empty or not, gets the next D_SID) are
// parsed on the host threads, every interval is keyed (shard * 64 + layer_for_size) << 32 | start
// and the keys are radix sorted on the device (LSD radix sort is stable, so equal starts keep file
// and line order).  Each (shard, layer) bucket then merges into the base index's layer with
// DeviceMerge: new elements first on equal starts, which is the order the reference's reverse
// co-merge writes (extend_layer, src/io/layer.rs:129-199: from the back, an old element is taken
// when old.start >= new.start, so old lands after new on ties).
//
// write: meta.json (serde field names of Meta, src/io/meta.rs:99-110), and per layer
// shards/<shard>/layer_K.{pos,sid,idx}: raw little-endian (start, end) u32 pairs, u32 sids, and the
// jump table as a flat u64 array (write_jump_table, src/io/jump.rs:116-133) holding, for tile t in
// 0..=max_start / tile_size, the partition point of start < t * tile_size — the table
// build_jump_table (src/io/jump.rs:66-115) computes for a freshly written layer.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <sys/stat.h>

#include "internal.h"

namespace rgl {
namespace {

__device__ __forceinline__ uint32_t dev_layer_for_size(uint32_t min_size, uint32_t gf, uint32_t size) {
    // LayerConfig::layer_for_size (src/io/meta.rs:33-58)
    if (size < min_size) return 0;
    uint64_t thr = min_size;
    uint32_t K = 0;
    while (thr <= size) {
        thr = thr > 0xFFFFFFFFFFFFFFFFull / gf ? 0xFFFFFFFFFFFFFFFFull : thr * gf;
        K++;
    }
    return K;
}

constexpr uint32_t kSlots = 64;  // layer slots per shard in the bucket key

__global__ void k_build_keys(uint64_t n, const rgl_interval* __restrict__ iv, const uint32_t* __restrict__ shard_of,
                             uint32_t min_size, uint32_t gf, uint64_t* __restrict__ key, uint32_t* __restrict__ val,
                             unsigned long long* __restrict__ hist, uint32_t* __restrict__ err) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const rgl_interval v = iv[i];
    uint32_t K = dev_layer_for_size(min_size, gf, v.end - v.start);
    if (K >= kSlots) {
        atomicOr(err, 1u);
        K = kSlots - 1;
    }
    const uint64_t b = (uint64_t)shard_of[i] * kSlots + K;
    key[i] = (b << 32) | v.start;
    val[i] = (uint32_t)i;
    atomicAdd(&hist[b], 1ull);
}

__global__ void k_new_starts(uint64_t n, const uint32_t* __restrict__ idx, const rgl_interval* __restrict__ iv,
                             uint32_t* __restrict__ out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = iv[idx[i]].start;
}

__global__ void k_base_starts(uint64_t n, const uint2* __restrict__ pos, uint32_t* __restrict__ out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = pos[i].x;
}

// v < new_n: new element idx[v] of the parsed intervals; else base element v - new_n.
__global__ void k_gather(uint64_t n, const uint32_t* __restrict__ order, uint64_t new_n,
                         const uint32_t* __restrict__ idx, const rgl_interval* __restrict__ iv,
                         const uint2* __restrict__ base_pos, const uint32_t* __restrict__ base_sid,
                         uint2* __restrict__ out_pos, uint32_t* __restrict__ out_sid) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t v = order ? order[i] : i;
    if (v < new_n) {
        const rgl_interval x = iv[idx[v]];
        out_pos[i] = make_uint2(x.start, x.end);
        out_sid[i] = x.sid;
    } else {
        out_pos[i] = base_pos[v - new_n];
        out_sid[i] = base_sid[v - new_n];
    }
}

inline unsigned grid(uint64_t n) { return (unsigned)((n + 255) / 256); }

bool ends_with(const std::string& s, const char* suf) {
    const size_t n = strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

std::string json_escape(const std::string& s) {
    std::string o;
    for (unsigned char c : s) {
        if (c == '"' || c == '\\') {
            o += '\\';
            o += (char)c;
        } else if (c < 0x20) {
            char b[8];
            snprintf(b, sizeof b, "\\u%04x", c);
            o += b;
        } else {
            o += (char)c;
        }
    }
    return o;
}

int mkdir_p(const std::string& path) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); i++) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
                return fail(RGL_ERR_IO, "cannot create directory " + cur);
        }
        if (i < path.size()) cur += path[i];
    }
    return RGL_OK;
}

int write_all(const std::string& path, const void* data, size_t bytes) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return fail(RGL_ERR_IO, "cannot write " + path);
    const size_t w = bytes ? fwrite(data, 1, bytes, f) : 0;
    const int c = fclose(f);
    if (w != bytes || c != 0) return fail(RGL_ERR_IO, "short write to " + path);
    return RGL_OK;
}

}  // namespace
}  // namespace rgl

using namespace rgl;

extern "C" {

int rgl_index_add_beds(const rgl_index* base, const char* input_path, uint32_t min_size, uint32_t gf,
                       uint32_t threads, int device, rgl_index** out) {
    clear_error();
    if (!input_path || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (base) {
        min_size = base->min_size;
        gf = base->gf;
        device = base->device;
    }
    if (min_size == 0 || gf < 2) return fail(RGL_ERR_INVALID_ARGUMENT, "layer_config needs min_size >= 1, growth_factor >= 2");
    std::vector<std::string> paths;
    bool is_dir = false;
    RGL_TRY(bed_list(input_path, &paths, &is_dir));
    if (!is_dir && !ends_with(paths[0], ".bed") && !ends_with(paths[0], ".bed.gz")) paths.clear();
    if (paths.empty()) return fail(RGL_ERR_NO_BED_FILES, std::string("No BED files found in ") + input_path);
    const uint32_t next_sid = base ? base->num_sources : 0;  // Meta::next_sid over contiguous sids
    std::vector<BedFile> files;
    RGL_TRY(bed_read_all(paths, next_sid, threads, &files));

    // shard ids: the base's, then new names in first-appearance order (files by path)
    std::vector<std::string> names = base ? base->shard_names : std::vector<std::string>();
    std::unordered_map<std::string, uint32_t> ids = base ? base->shard_ids : std::unordered_map<std::string, uint32_t>();
    uint64_t n = 0;
    for (auto& f : files)
        for (size_t k = 0; k < f.shards.size(); k++) {
            if (!ids.count(f.shards[k])) {
                ids[f.shards[k]] = (uint32_t)names.size();
                names.push_back(f.shards[k]);
            }
            n += f.ivs[k].size();
        }
    if (n >= (1ull << 31)) return fail(RGL_ERR_UNSUPPORTED, "at most 2^31 - 1 intervals per add");
    const uint32_t S = (uint32_t)names.size();
    std::vector<rgl_interval> iv;
    std::vector<uint32_t> shard_of;
    iv.reserve(n);
    shard_of.reserve(n);
    for (auto& f : files)
        for (size_t k = 0; k < f.shards.size(); k++) {
            iv.insert(iv.end(), f.ivs[k].begin(), f.ivs[k].end());
            shard_of.insert(shard_of.end(), f.ivs[k].size(), ids[f.shards[k]]);
        }
    RGL_CUDA(cudaSetDevice(device));
    const uint64_t nb = (uint64_t)std::max<uint32_t>(S, 1) * kSlots;
    DevBuf d_iv, d_shard, ka, kb, va, vb, d_hist, d_err, tmp;
    int s = RGL_OK;
    const uint64_t nn = std::max<uint64_t>(n, 1);
    for (auto& x : std::initializer_list<std::pair<DevBuf*, size_t>>{
             {&d_iv, nn * sizeof(rgl_interval)}, {&d_shard, nn * 4}, {&ka, nn * 8}, {&kb, nn * 8}, {&va, nn * 4},
             {&vb, nn * 4}, {&d_hist, nb * 8}, {&d_err, 16}})
        if (s == RGL_OK) s = x.first->ensure(x.second);
    int kbits = 1;
    while ((1ull << kbits) < nb) kbits++;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint64_t*)nullptr, (uint64_t*)nullptr, (uint32_t*)nullptr,
                                    (uint32_t*)nullptr, (int)nn, 0, 32 + kbits);
    if (s == RGL_OK) s = tmp.ensure(tb + 256);
    std::vector<unsigned long long> hist(nb, 0);
    uint32_t err = 0;
    if (s == RGL_OK && n) {
        if (cudaMemcpy(d_iv.p, iv.data(), n * sizeof(rgl_interval), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_shard.p, shard_of.data(), n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(d_hist.p, 0, nb * 8) != cudaSuccess || cudaMemset(d_err.p, 0, 4) != cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "index build upload");
        if (s == RGL_OK) {
            k_build_keys<<<grid(n), 256>>>(n, d_iv.as<rgl_interval>(), d_shard.as<uint32_t>(), min_size, gf,
                                           ka.as<uint64_t>(), va.as<uint32_t>(), d_hist.as<unsigned long long>(),
                                           d_err.as<uint32_t>());
            size_t t2 = tmp.cap;
            if (cub::DeviceRadixSort::SortPairs(tmp.p, t2, ka.as<uint64_t>(), kb.as<uint64_t>(), va.as<uint32_t>(),
                                                vb.as<uint32_t>(), (int)n, 0, 32 + kbits) != cudaSuccess ||
                cudaMemcpy(hist.data(), d_hist.p, nb * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(&err, d_err.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
                s = fail(RGL_ERR_DEVICE, "index build sort");
        }
        if (s == RGL_OK && err) s = fail(RGL_ERR_UNSUPPORTED, "an interval falls in a layer >= 64");
    }
    // the merged layer table, ordered by (shard, layer)
    auto* idx = new rgl_index();
    idx->device = device;
    idx->min_size = min_size;
    idx->gf = gf;
    idx->num_sources = next_sid + (uint32_t)files.size();
    idx->num_shards = S;
    idx->shard_names = names;
    idx->shard_ids = ids;
    if (base) idx->source_names = base->source_names;
    for (auto& f : files) idx->source_names.push_back(f.name);
    std::vector<uint64_t> new_off(nb + 1, 0);
    for (uint64_t b = 0; b < nb; b++) new_off[b + 1] = new_off[b] + hist[b];
    struct Src { int64_t base_layer; uint64_t new_n, new_at; };
    std::vector<Src> srcs;
    for (uint32_t sh = 0; sh < S && s == RGL_OK; sh++)
        for (uint32_t K = 0; K < kSlots; K++) {
            int64_t bl = -1;
            if (base && sh < base->num_shards && K < base->num_slots) bl = base->slot[(size_t)sh * base->num_slots + K];
            const uint64_t bn = bl >= 0 ? base->layers[bl].n : 0, nw = hist[(uint64_t)sh * kSlots + K];
            if (!bn && !nw) continue;
            LayerDev l{};
            l.n = bn + nw;
            l.shard = sh;
            l.layer = K;
            l.max_size = layer_max_size(min_size, gf, K);
            idx->layers.push_back(l);
            idx->total += l.n;
            srcs.push_back(Src{bl, nw, new_off[(uint64_t)sh * kSlots + K]});
        }
    uint32_t maxk = 0;
    for (auto& l : idx->layers) maxk = std::max(maxk, l.layer + 1);
    idx->num_slots = maxk;
    idx->slot.assign((size_t)S * maxk, -1);
    for (size_t i = 0; i < idx->layers.size(); i++)
        idx->slot[(size_t)idx->layers[i].shard * maxk + idx->layers[i].layer] = (int32_t)i;
    if (s == RGL_OK) s = index_alloc(idx);
    // per layer: copy, gather or merge
    uint64_t mx = 1;
    for (auto& l : idx->layers) mx = std::max(mx, l.n);
    if (s == RGL_OK && mx >= (1ull << 31)) s = fail(RGL_ERR_UNSUPPORTED, "a merged layer of 2^31 or more intervals");
    DevBuf k1, k2, mk, mv, mtmp;
    if (s == RGL_OK) s = k1.ensure(mx * 4);
    if (s == RGL_OK) s = k2.ensure(mx * 4);
    if (s == RGL_OK) s = mk.ensure(mx * 4);
    if (s == RGL_OK) s = mv.ensure(mx * 4);
    for (size_t i = 0; i < idx->layers.size() && s == RGL_OK; i++) {
        const LayerDev& L = idx->layers[i];
        const Src& sc = srcs[i];
        uint2* op = idx->d_pos + L.off;
        uint32_t* os = idx->d_sid + L.off;
        const uint32_t* nidx = vb.as<uint32_t>() + sc.new_at;
        const LayerDev* BL = sc.base_layer >= 0 ? &base->layers[sc.base_layer] : nullptr;
        if (!BL) {
            k_gather<<<grid(L.n), 256>>>(L.n, nullptr, sc.new_n, nidx, d_iv.as<rgl_interval>(), nullptr, nullptr, op, os);
        } else if (!sc.new_n) {
            if (cudaMemcpy(op, base->d_pos + BL->off, BL->n * 8, cudaMemcpyDeviceToDevice) != cudaSuccess ||
                cudaMemcpy(os, base->d_sid + BL->off, BL->n * 4, cudaMemcpyDeviceToDevice) != cudaSuccess)
                s = fail(RGL_ERR_DEVICE, "layer copy");
        } else {
            k_new_starts<<<grid(sc.new_n), 256>>>(sc.new_n, nidx, d_iv.as<rgl_interval>(), k1.as<uint32_t>());
            k_base_starts<<<grid(BL->n), 256>>>(BL->n, base->d_pos + BL->off, k2.as<uint32_t>());
            // new first on equal starts: the first input wins ties
            thrust::counting_iterator<uint32_t> v1(0), v2((uint32_t)sc.new_n);
            size_t t3 = 0;
            cub::DeviceMerge::MergePairs(nullptr, t3, k1.as<uint32_t>(), v1, (int)sc.new_n, k2.as<uint32_t>(), v2,
                                         (int)BL->n, mk.as<uint32_t>(), mv.as<uint32_t>());
            if ((s = mtmp.ensure(t3 + 256)) != RGL_OK) break;
            t3 = mtmp.cap;
            if (cub::DeviceMerge::MergePairs(mtmp.p, t3, k1.as<uint32_t>(), v1, (int)sc.new_n, k2.as<uint32_t>(), v2,
                                             (int)BL->n, mk.as<uint32_t>(), mv.as<uint32_t>()) != cudaSuccess) {
                s = fail(RGL_ERR_DEVICE, "layer merge");
                break;
            }
            k_gather<<<grid(L.n), 256>>>(L.n, mv.as<uint32_t>(), sc.new_n, nidx, d_iv.as<rgl_interval>(),
                                         base->d_pos + BL->off, base->d_sid + BL->off, op, os);
        }
        if (s == RGL_OK && cudaGetLastError() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "index build kernels");
    }
    if (s == RGL_OK && cudaDeviceSynchronize() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "index build");
    for (DevBuf* b : {&d_iv, &d_shard, &ka, &kb, &va, &vb, &d_hist, &d_err, &tmp, &k1, &k2, &mk, &mv, &mtmp}) b->release();
    if (s == RGL_OK) s = index_finalize(idx);
    if (s != RGL_OK) {
        index_free(idx);
        delete idx;
        return s;
    }
    *out = idx;
    return RGL_OK;
}

int rgl_index_write(const rgl_index* idx, const char* db_dir) {
    clear_error();
    if (!idx || !db_dir) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    const std::string root(db_dir);
    RGL_TRY(mkdir_p(root + "/shards"));
    RGL_CUDA(cudaSetDevice(idx->device));
    uint32_t num_layers = 0;
    std::vector<uint32_t> pos;
    std::vector<uint32_t> sid;
    for (const LayerDev& L : idx->layers) {
        num_layers = std::max(num_layers, L.layer + 1);
        const std::string dir = root + "/shards/" + idx->shard_names[L.shard];
        RGL_TRY(mkdir_p(dir));
        pos.resize(2 * L.n);
        sid.resize(L.n);
        RGL_CUDA(cudaMemcpy(pos.data(), idx->d_pos + L.off, L.n * 8, cudaMemcpyDeviceToHost));
        RGL_CUDA(cudaMemcpy(sid.data(), idx->d_sid + L.off, L.n * 4, cudaMemcpyDeviceToHost));
        const std::string stem = dir + "/layer_" + std::to_string(L.layer);
        RGL_TRY(write_all(stem + ".pos", pos.data(), L.n * 8));
        RGL_TRY(write_all(stem + ".sid", sid.data(), L.n * 4));
        const uint64_t tile = tile_size(idx->min_size, idx->gf, L.layer);
        std::vector<uint64_t> jt(1, 0);
        if (L.n) {
            const uint64_t max_tile = pos[2 * (L.n - 1)] / tile;
            jt.assign(max_tile + 1, 0);
            uint64_t j = 0;
            for (uint64_t t = 0; t <= max_tile; t++) {
                while (j < L.n && (uint64_t)pos[2 * j] < t * tile) j++;
                jt[t] = j;
            }
        }
        RGL_TRY(write_all(stem + ".idx", jt.data(), jt.size() * 8));
    }
    std::string js = "{\n  \"sid_map\": {";
    for (uint32_t d = 0; d < idx->num_sources; d++)
        js += std::string(d ? "," : "") + "\n    \"" + std::to_string(d) + "\": {\n      \"name\": \"" +
              json_escape(d < idx->source_names.size() ? idx->source_names[d] : "source_" + std::to_string(d)) +
              "\"\n    }";
    js += std::string(idx->num_sources ? "\n  " : "") + "},\n  \"layer_config\": {\n    \"min_size\": " +
          std::to_string(idx->min_size) + ",\n    \"growth_factor\": " + std::to_string(idx->gf) + "\n  },\n  \"shards\": [";
    for (uint32_t s = 0; s < idx->num_shards; s++)
        js += std::string(s ? "," : "") + "\n    \"" + json_escape(idx->shard_names[s]) + "\"";
    js += std::string(idx->num_shards ? "\n  " : "") + "],\n  \"num_layers\": " + std::to_string(num_layers) + "\n}";
    return write_all(root + "/meta.json", js.data(), js.size());
}

}  // extern "C"
