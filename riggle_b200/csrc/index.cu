// Device-resident database index: the reference's per-(shard, layer) `.pos` / `.sid` arrays
// (src/io/layer.rs:31-105) copied into two index-wide HBM arrays, plus a layer table.
//
// HBM layout: d_pos is uint2[(start, end)] exactly as layer_K.pos stores it, d_sid is u32 as in
// layer_K.sid; layer l occupies elements [off_l, off_l + n_l) of both, with off_l a multiple of 4
// (16-byte aligned sid blocks, 32-byte aligned pos blocks).  The reference's `.idx` jump table
// (src/io/jump.rs) is size-checked at open for error parity but not uploaded: the device computes
// exact partition points by binary search, which is what the reference's conservative lookup plus
// partition_point yields (src/sweep/query.rs:98-100).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "internal.h"

namespace rgl {

int DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return RGL_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        return fail(RGL_ERR_OOM, std::string("cudaMalloc(") + std::to_string(want) + "): " + cudaGetErrorString(e));
    }
    cap = want;
    return RGL_OK;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

__global__ void k_validate_layer(const uint2* __restrict__ pos, const uint32_t* __restrict__ sid, uint64_t n,
                                 uint32_t max_size, uint32_t num_sources, uint32_t* __restrict__ flags) {
    uint32_t f = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint2 p = pos[i];
        if (p.x >= p.y) f |= LF_EMPTY_IV;
        else if (p.y - p.x >= max_size) f |= LF_OVERSIZE;
        if (i > 0 && pos[i - 1].x > p.x) f |= LF_UNSORTED;
        if (sid[i] >= num_sources) f |= LF_BAD_SID;
    }
    f = __reduce_or_sync(0xffffffffu, f);
    if (f && (threadIdx.x & 31) == 0) atomicOr(flags, f);
}

// Bucket table of one sorted layer: thread j writes j into the buckets after element j-1's bucket
// up to its own (j == n: up to the last entry), so tab[b] = first j with start_j >= b << s.
__global__ void k_bucket_fill(const uint2* __restrict__ pos, uint64_t n, uint32_t s, uint32_t nb,
                              uint32_t* __restrict__ tab) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j <= n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t lo_b = j == 0 ? 0u : (pos[j - 1].x >> s) + 1u;
        const uint32_t hi_b = j == n ? nb - 1u : (pos[j].x >> s);
        for (uint32_t b = lo_b; b <= hi_b && b < nb; b++) tab[b] = (uint32_t)j;
    }
}

int index_alloc(rgl_index* idx) {
    uint64_t off = 0;
    for (auto& l : idx->layers)
        if (l.n >= 0xFFFFFFFFull)
            return fail(RGL_ERR_UNSUPPORTED, "a layer holds 2^32-1 or more intervals (layer indices are 32-bit)");
    for (auto& l : idx->layers) {
        l.off = off;
        off += (l.n + 3) & ~uint64_t(3);
    }
    idx->cap_elems = off < 4 ? 4 : off;
    RGL_CUDA(cudaSetDevice(idx->device));
    RGL_CUDA(cudaMalloc(&idx->d_pos, idx->cap_elems * sizeof(uint2)));
    RGL_CUDA(cudaMalloc(&idx->d_sid, idx->cap_elems * sizeof(uint32_t)));
    idx->device_bytes = idx->cap_elems * 12;
    return RGL_OK;
}

int index_finalize(rgl_index* idx) {
    RGL_CUDA(cudaSetDevice(idx->device));
    size_t nl = idx->layers.size() ? idx->layers.size() : 1;
    RGL_CUDA(cudaMalloc(&idx->d_layers, nl * sizeof(LayerDev)));
    size_t ns = idx->slot.size() ? idx->slot.size() : 1;
    RGL_CUDA(cudaMalloc(&idx->d_slot, ns * sizeof(int32_t)));
    idx->device_bytes += nl * sizeof(LayerDev) + ns * sizeof(int32_t);
    uint32_t* d_flags = nullptr;
    RGL_CUDA(cudaMalloc(&d_flags, nl * sizeof(uint32_t)));
    RGL_CUDA(cudaMemset(d_flags, 0, nl * sizeof(uint32_t)));
    for (size_t i = 0; i < idx->layers.size(); i++) {
        const LayerDev& l = idx->layers[i];
        uint64_t blocks = (l.n + 255) / 256;
        if (blocks > 148 * 16) blocks = 148 * 16;
        if (blocks == 0) blocks = 1;
        k_validate_layer<<<(unsigned)blocks, 256>>>(idx->d_pos + l.off, idx->d_sid + l.off, l.n, l.max_size,
                                                     idx->num_sources, d_flags + i);
    }
    RGL_CUDA(cudaGetLastError());
    std::vector<uint32_t> flags(nl, 0);
    RGL_CUDA(cudaMemcpy(flags.data(), d_flags, nl * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    cudaFree(d_flags);
    for (size_t i = 0; i < idx->layers.size(); i++) {
        LayerDev& l = idx->layers[i];
        l.flags = flags[i];
        std::string where = "shard '" + idx->shard_names[l.shard] + "' layer " + std::to_string(l.layer);
        if (l.flags & LF_UNSORTED)
            return fail(RGL_ERR_INDEX_INVARIANT, where + ": positions are not sorted by start");
        if (l.flags & LF_BAD_SID)
            return fail(RGL_ERR_INDEX_INVARIANT,
                        where + ": a source id is >= num_sources (" + std::to_string(idx->num_sources) + ")");
        if (l.flags & (LF_EMPTY_IV | LF_OVERSIZE))
            return fail(RGL_ERR_INDEX_INVARIANT,
                        where + ": an interval has start >= end or a size outside its layer's class "
                                "(the reference's add never writes one)");
    }
    // bucket tables: widths 2^s >= (max start + 1) / n, so about one interval per bucket and at most
    // n + 2 entries (4 bytes per interval)
    uint64_t btot = 0;
    for (LayerDev& l : idx->layers) {
        uint32_t maxstart = 0;
        if (l.n) RGL_CUDA(cudaMemcpy(&maxstart, &idx->d_pos[l.off + l.n - 1].x, 4, cudaMemcpyDeviceToHost));
        const uint64_t ratio = l.n ? ((uint64_t)maxstart + 1 + l.n - 1) / l.n : 1;
        uint32_t sh = 0;
        while (sh < 31 && (1ull << sh) < ratio) sh++;
        l.bshift = sh;
        l.nb = (maxstart >> sh) + 2;
        l.boff = btot;
        btot += l.nb;
    }
    if (idx->d_btab) cudaFree(idx->d_btab);
    idx->d_btab = nullptr;
    RGL_CUDA(cudaMalloc(&idx->d_btab, std::max<uint64_t>(btot, 1) * 4));
    idx->device_bytes += std::max<uint64_t>(btot, 1) * 4;
    for (const LayerDev& l : idx->layers) {
        const unsigned blocks = (unsigned)std::min<uint64_t>((l.n + 256) / 256, 148ull * 32);
        k_bucket_fill<<<blocks, 256>>>(idx->d_pos + l.off, l.n, l.bshift, l.nb, idx->d_btab + l.boff);
    }
    RGL_CUDA(cudaGetLastError());
    RGL_CUDA(cudaDeviceSynchronize());
    if (!idx->layers.empty())
        RGL_CUDA(cudaMemcpy(idx->d_layers, idx->layers.data(), idx->layers.size() * sizeof(LayerDev),
                            cudaMemcpyHostToDevice));
    if (!idx->slot.empty())
        RGL_CUDA(cudaMemcpy(idx->d_slot, idx->slot.data(), idx->slot.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    return RGL_OK;
}

void index_release(rgl_index* idx) {
    if (idx && idx->refs.fetch_sub(1) == 1) {
        index_free(idx);
        delete idx;
    }
}

void index_free(rgl_index* idx) {
    if (!idx) return;
    cudaSetDevice(idx->device);
    if (idx->d_pos) cudaFree(idx->d_pos);
    if (idx->d_sid) cudaFree(idx->d_sid);
    if (idx->d_layers) cudaFree(idx->d_layers);
    if (idx->d_btab) cudaFree(idx->d_btab);
    idx->d_btab = nullptr;
    if (idx->d_slot) cudaFree(idx->d_slot);
    idx->d_pos = nullptr;
    idx->d_sid = nullptr;
    idx->d_layers = nullptr;
    idx->d_slot = nullptr;
}

static int check_layer_config(uint32_t min_size, uint32_t gf) {
    if (min_size == 0 || gf < 2)
        return fail(RGL_ERR_INVALID_ARGUMENT, "layer_config needs min_size >= 1 and growth_factor >= 2 (min_size=" +
                                                  std::to_string(min_size) + ", growth_factor=" + std::to_string(gf) + ")");
    return RGL_OK;
}

static int device_check(int device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(RGL_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= n) return fail(RGL_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    return RGL_OK;
}

// Column filter: flag[i] = sid in [lo, hi); after an exclusive scan, the kept elements move to
// their compacted positions in order (so every layer stays sorted by start), sids rebased to 0.
__global__ void k_col_flags(const uint32_t* __restrict__ sid, uint64_t n, uint32_t lo, uint32_t hi,
                            uint32_t* __restrict__ flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = (i < n && sid[i] >= lo && sid[i] < hi) ? 1u : 0u;
}

__global__ void k_col_scatter(const uint2* __restrict__ pos, const uint32_t* __restrict__ sid, uint64_t n,
                              const uint32_t* __restrict__ flag, const uint32_t* __restrict__ at, uint32_t lo,
                              uint2* __restrict__ out_pos, uint32_t* __restrict__ out_sid) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i]) {
            out_pos[at[i]] = pos[i];
            out_sid[at[i]] = sid[i] - lo;
        }
}

}  // namespace rgl

using namespace rgl;

// Builds the shard/slot tables of an index from its (shard, layer, n) triples.
static void build_slots(rgl_index* idx) {
    uint32_t maxk = 0;
    for (auto& l : idx->layers) maxk = std::max(maxk, l.layer + 1);
    idx->num_slots = maxk;
    idx->slot.assign((size_t)idx->num_shards * maxk, -1);
    for (size_t i = 0; i < idx->layers.size(); i++)
        idx->slot[(size_t)idx->layers[i].shard * maxk + idx->layers[i].layer] = (int32_t)i;
}

extern "C" {

int rgl_index_open_mem(const rgl_index_desc* desc, int device, rgl_index** out) {
    clear_error();
    if (!desc || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    RGL_TRY(check_layer_config(desc->min_size, desc->growth_factor));
    RGL_TRY(device_check(device));
    auto* idx = new rgl_index();
    idx->device = device;
    idx->min_size = desc->min_size;
    idx->gf = desc->growth_factor;
    idx->num_sources = desc->num_sources;
    idx->num_shards = desc->num_shards;
    for (uint32_t s = 0; s < desc->num_shards; s++) {
        std::string nm = desc->shard_names && desc->shard_names[s] ? desc->shard_names[s] : std::to_string(s);
        idx->shard_names.push_back(nm);
        idx->shard_ids[nm] = s;
    }
    for (uint32_t d = 0; d < desc->num_sources; d++)
        idx->source_names.push_back(desc->source_names && desc->source_names[d] ? desc->source_names[d]
                                                                               : "source_" + std::to_string(d));
    for (uint32_t i = 0; i < desc->num_layers; i++) {
        const rgl_layer_desc& ld = desc->layers[i];
        if (ld.shard >= desc->num_shards) {
            delete idx;
            return fail(RGL_ERR_INVALID_ARGUMENT, "layer descriptor names shard " + std::to_string(ld.shard));
        }
        if (ld.count == 0) continue;
        if (!ld.pos || !ld.sid) {
            delete idx;
            return fail(RGL_ERR_INVALID_ARGUMENT, "layer descriptor without pos/sid arrays");
        }
        for (auto& l : idx->layers)
            if (l.shard == ld.shard && l.layer == ld.layer) {
                delete idx;
                return fail(RGL_ERR_INVALID_ARGUMENT, "duplicate (shard, layer) descriptor");
            }
        LayerDev l{};
        l.n = ld.count;
        l.shard = ld.shard;
        l.layer = ld.layer;
        l.max_size = layer_max_size(desc->min_size, desc->growth_factor, ld.layer);
        idx->layers.push_back(l);
        idx->total += ld.count;
    }
    build_slots(idx);
    int s = index_alloc(idx);
    if (s == RGL_OK) {
        size_t li = 0;
        for (uint32_t i = 0; i < desc->num_layers && s == RGL_OK; i++) {
            const rgl_layer_desc& ld = desc->layers[i];
            if (ld.count == 0) continue;
            const LayerDev& l = idx->layers[li++];
            cudaError_t e1 = cudaMemcpy(idx->d_pos + l.off, ld.pos, l.n * 8, cudaMemcpyHostToDevice);
            cudaError_t e2 = cudaMemcpy(idx->d_sid + l.off, ld.sid, l.n * 4, cudaMemcpyHostToDevice);
            if (e1 != cudaSuccess || e2 != cudaSuccess)
                s = fail(RGL_ERR_DEVICE, std::string("layer upload: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        }
    }
    if (s == RGL_OK) s = index_finalize(idx);
    if (s != RGL_OK) {
        index_free(idx);
        delete idx;
        return s;
    }
    *out = idx;
    return RGL_OK;
}

int rgl_index_open(const char* db_dir, int device, rgl_index** out) {
    clear_error();
    if (!db_dir || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::string dir(db_dir);
    // query_database returns DatabaseNotFound when meta.json is absent (src/tasks/query/mod.rs:124-127).
    if (!file_exists(dir + "/meta.json")) return fail(RGL_ERR_DATABASE_NOT_FOUND, "Database not found at " + dir);
    MetaInfo meta;
    RGL_TRY(meta_load(dir, &meta));
    RGL_TRY(check_layer_config(meta.min_size, meta.growth_factor));
    RGL_TRY(device_check(device));

    auto* idx = new rgl_index();
    idx->device = device;
    idx->min_size = meta.min_size;
    idx->gf = meta.growth_factor;
    idx->num_sources = (uint32_t)meta.sid_map.size();  // Meta::num_sources (src/io/meta.rs:142-144)
    idx->num_shards = (uint32_t)meta.shards.size();
    for (uint32_t s = 0; s < idx->num_shards; s++) {
        idx->shard_names.push_back(meta.shards[s]);
        idx->shard_ids[meta.shards[s]] = s;
    }
    for (uint32_t d = 0; d < idx->num_sources; d++) {
        auto it = meta.sid_map.find(d);
        idx->source_names.push_back(it != meta.sid_map.end() ? it->second : "source_" + std::to_string(d));
    }
    struct Pending {
        std::string pos, sid;
    };
    std::vector<Pending> files;
    int s = RGL_OK;
    // Same file checks and order as query_database's layer loading (src/tasks/query/mod.rs:205-233)
    // and MappedLayer::open / MappedJumpTable::open (src/io/layer.rs:51-78, src/io/jump.rs:27-44).
    for (uint32_t sh = 0; sh < idx->num_shards && s == RGL_OK; sh++) {
        for (uint64_t k = 0; k < meta.num_layers && s == RGL_OK; k++) {
            std::string base = dir + "/shards/" + meta.shards[sh] + "/layer_" + std::to_string(k);
            if (!file_exists(base + ".pos")) continue;
            FILE* fp = std::fopen((base + ".pos").c_str(), "rb");
            FILE* fs = std::fopen((base + ".sid").c_str(), "rb");
            if (!fp || !fs) {
                if (fp) std::fclose(fp);
                if (fs) std::fclose(fs);
                s = fail(RGL_ERR_IO, "cannot open " + base + (fp ? ".sid" : ".pos"));
                break;
            }
            std::fseek(fp, 0, SEEK_END);
            std::fseek(fs, 0, SEEK_END);
            uint64_t psz = (uint64_t)std::ftell(fp), ssz = (uint64_t)std::ftell(fs);
            std::fclose(fp);
            std::fclose(fs);
            if (psz % 8) { s = fail(RGL_ERR_LAYER_INVALID_POSITION_SIZE, "Position file has invalid size: " + std::to_string(psz) + " bytes"); break; }
            if (ssz % 4) { s = fail(RGL_ERR_LAYER_INVALID_SID_SIZE, "Sid file has invalid size: " + std::to_string(ssz) + " bytes"); break; }
            if (psz / 8 != ssz / 4) {
                s = fail(RGL_ERR_LAYER_SID_SIZE_MISMATCH, "Position count " + std::to_string(psz / 8) +
                                                              " does not match sid count " + std::to_string(ssz / 4));
                break;
            }
            if (psz == 0) continue;  // empty layers are skipped before the jump table is opened
            FILE* fi = std::fopen((base + ".idx").c_str(), "rb");
            if (!fi) { s = fail(RGL_ERR_IO, "cannot open " + base + ".idx"); break; }
            std::fseek(fi, 0, SEEK_END);
            uint64_t isz = (uint64_t)std::ftell(fi);
            std::fclose(fi);
            if (isz % 8) { s = fail(RGL_ERR_LAYER_INVALID_INDEX_SIZE, "Index file has invalid size: " + std::to_string(isz) + " bytes (not a multiple of 4)"); break; }
            LayerDev l{};
            l.n = psz / 8;
            l.shard = sh;
            l.layer = (uint32_t)k;
            l.max_size = layer_max_size(meta.min_size, meta.growth_factor, (uint32_t)k);
            idx->layers.push_back(l);
            idx->total += l.n;
            files.push_back({base + ".pos", base + ".sid"});
        }
    }
    if (s == RGL_OK) {
        build_slots(idx);
        s = index_alloc(idx);
    }
    // Stream the files through a pinned staging buffer.
    if (s == RGL_OK && !files.empty()) {
        const size_t CH = 64u << 20;
        void* stage = nullptr;
        if (cudaMallocHost(&stage, CH) != cudaSuccess) s = fail(RGL_ERR_OOM, "pinned staging buffer");
        for (size_t i = 0; i < files.size() && s == RGL_OK; i++) {
            const LayerDev& l = idx->layers[i];
            for (int which = 0; which < 2 && s == RGL_OK; which++) {
                const std::string& path = which == 0 ? files[i].pos : files[i].sid;
                uint8_t* dst = which == 0 ? reinterpret_cast<uint8_t*>(idx->d_pos + l.off)
                                          : reinterpret_cast<uint8_t*>(idx->d_sid + l.off);
                uint64_t bytes = l.n * (which == 0 ? 8 : 4);
                FILE* f = std::fopen(path.c_str(), "rb");
                if (!f) { s = fail(RGL_ERR_IO, "cannot open " + path); break; }
                uint64_t done = 0;
                while (done < bytes) {
                    size_t want = (size_t)std::min<uint64_t>(CH, bytes - done);
                    size_t got = std::fread(stage, 1, want, f);
                    if (got != want) { s = fail(RGL_ERR_IO, "short read of " + path); break; }
                    if (cudaMemcpy(dst + done, stage, got, cudaMemcpyHostToDevice) != cudaSuccess) {
                        s = fail(RGL_ERR_DEVICE, "layer upload failed");
                        break;
                    }
                    done += got;
                }
                std::fclose(f);
            }
        }
        if (stage) cudaFreeHost(stage);
    }
    if (s == RGL_OK) s = index_finalize(idx);
    if (s != RGL_OK) {
        index_free(idx);
        delete idx;
        return s;
    }
    *out = idx;
    return RGL_OK;
}

int rgl_index_close(rgl_index* index) {
    clear_error();
    index_release(index);
    return RGL_OK;
}

int rgl_index_get_info(const rgl_index* index, rgl_index_info* out) {
    if (!index || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    out->num_sources = index->num_sources;
    out->num_shards = index->num_shards;
    out->num_layer_slots = index->num_slots;
    out->num_layers = (uint32_t)index->layers.size();
    out->num_intervals = index->total;
    out->device_bytes = index->device_bytes;
    out->device = index->device;
    return RGL_OK;
}

int rgl_index_shard_id(const rgl_index* index, const char* name, uint32_t* out_id) {
    if (!index || !name || !out_id) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    auto it = index->shard_ids.find(name);
    if (it == index->shard_ids.end()) return fail(RGL_ERR_INVALID_ARGUMENT, std::string("shard not in index: ") + name);
    *out_id = it->second;
    return RGL_OK;
}

const char* rgl_index_shard_name(const rgl_index* index, uint32_t shard) {
    if (!index || shard >= index->num_shards) return nullptr;
    return index->shard_names[shard].c_str();
}

const char* rgl_index_source_name(const rgl_index* index, uint32_t sid) {
    if (!index || sid >= index->num_sources) return nullptr;
    return index->source_names[sid].c_str();
}

uint64_t rgl_index_layer_count(const rgl_index* index, uint32_t shard, uint32_t layer) {
    if (!index || shard >= index->num_shards || layer >= index->num_slots) return 0;
    int32_t li = index->slot[(size_t)shard * index->num_slots + layer];
    return li < 0 ? 0 : index->layers[li].n;
}

int rgl_index_export_layer(const rgl_index* index, uint32_t shard, uint32_t layer, uint32_t* pos, uint32_t* sid) {
    if (!index) return fail(RGL_ERR_INVALID_ARGUMENT, "null index");
    if (shard >= index->num_shards || layer >= index->num_slots) return RGL_OK;
    int32_t li = index->slot[(size_t)shard * index->num_slots + layer];
    if (li < 0) return RGL_OK;
    const LayerDev& l = index->layers[li];
    RGL_CUDA(cudaSetDevice(index->device));
    if (pos) RGL_CUDA(cudaMemcpy(pos, index->d_pos + l.off, l.n * 8, cudaMemcpyDeviceToHost));
    if (sid) RGL_CUDA(cudaMemcpy(sid, index->d_sid + l.off, l.n * 4, cudaMemcpyDeviceToHost));
    return RGL_OK;
}

int rgl_index_select_columns(const rgl_index* src, uint32_t sid_lo, uint32_t sid_hi, rgl_index** out) {
    clear_error();
    if (!src || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (sid_lo > sid_hi || sid_hi > src->num_sources) return fail(RGL_ERR_INVALID_ARGUMENT, "bad source range");
    RGL_CUDA(cudaSetDevice(src->device));
    uint64_t maxn = 1;
    for (auto& l : src->layers) maxn = std::max(maxn, l.n);
    DevBuf flag, at, tmp;
    int s = flag.ensure((maxn + 1) * 4);
    if (s == RGL_OK) s = at.ensure((maxn + 1) * 4);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)(maxn + 1));
    if (s == RGL_OK) s = tmp.ensure(tb + 256);
    if (s == RGL_OK && maxn + 1 >= (1ull << 31)) s = fail(RGL_ERR_UNSUPPORTED, "a layer of 2^31 or more intervals");
    // pass 1: kept count of every layer
    std::vector<uint64_t> kept(src->layers.size(), 0);
    auto run_flags = [&](const LayerDev& l) -> int {
        const unsigned blocks = (unsigned)std::min<uint64_t>((l.n + 256) / 256, 148ull * 16);
        k_col_flags<<<blocks, 256>>>(src->d_sid + l.off, l.n, sid_lo, sid_hi, flag.as<uint32_t>());
        size_t t = tmp.cap;
        RGL_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, t, flag.as<uint32_t>(), at.as<uint32_t>(), (int)(l.n + 1)));
        return RGL_OK;
    };
    for (size_t i = 0; i < src->layers.size() && s == RGL_OK; i++) {
        s = run_flags(src->layers[i]);
        uint32_t k = 0;
        if (s == RGL_OK && cudaMemcpy(&k, at.as<uint32_t>() + src->layers[i].n, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            s = fail(RGL_ERR_DEVICE, "column count");
        kept[i] = k;
    }
    auto* idx = new rgl_index();
    idx->device = src->device;
    idx->min_size = src->min_size;
    idx->gf = src->gf;
    idx->num_sources = sid_hi - sid_lo;
    idx->num_shards = src->num_shards;
    idx->shard_names = src->shard_names;
    idx->shard_ids = src->shard_ids;
    for (uint32_t d = sid_lo; d < sid_hi; d++) idx->source_names.push_back(src->source_names[d]);
    std::vector<size_t> from;
    for (size_t i = 0; i < src->layers.size(); i++)
        if (kept[i]) {
            LayerDev l = src->layers[i];
            l.n = kept[i];
            l.flags = 0;
            idx->layers.push_back(l);
            idx->total += l.n;
            from.push_back(i);
        }
    build_slots(idx);
    if (s == RGL_OK) s = index_alloc(idx);
    // pass 2: compaction into the new blocks
    for (size_t j = 0; j < idx->layers.size() && s == RGL_OK; j++) {
        const LayerDev& l = src->layers[from[j]];
        s = run_flags(l);
        if (s != RGL_OK) break;
        const unsigned blocks = (unsigned)std::min<uint64_t>((l.n + 255) / 256, 148ull * 16);
        k_col_scatter<<<blocks, 256>>>(src->d_pos + l.off, src->d_sid + l.off, l.n, flag.as<uint32_t>(),
                                       at.as<uint32_t>(), sid_lo, idx->d_pos + idx->layers[j].off,
                                       idx->d_sid + idx->layers[j].off);
        if (cudaGetLastError() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "column scatter");
    }
    if (s == RGL_OK && cudaDeviceSynchronize() != cudaSuccess) s = fail(RGL_ERR_DEVICE, "column filter");
    flag.release();
    at.release();
    tmp.release();
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
