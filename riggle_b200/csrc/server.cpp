// Request server: continuous batching of query files against a resident index.
//
// Worker threads each own a query context (its own CUDA stream and workspace), a device staging
// buffer for the intervals of one batch, device and page-locked output rows and, with a moment
// store, their own scratch for the stats stage.  An idle worker takes the oldest pending requests
// as one batch: one host-to-device copy per request, one pipeline run with the rows taken from the
// blocks, the p-values of the batch's rows when the server has a moment store, one device-to-host
// copy of each output, then the rows are handed to their requests.  With several workers, requests
// that arrive while a batch is on the GPU start on another stream at once, so their work overlaps on
// the device.
//
// Admission by free device memory happens when a batch is formed: a worker starts with a modest
// workspace and a request joins its batch only while the memory the batch would add to the worker
// (workspace, staging and output growth, computed without allocating) fits in the free memory less
// the reserve and less what other workers have been promised but not yet allocated.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "block_sort.cuh"
#include "internal.h"

namespace rgl {
namespace {

struct Req {
    rgl_request r;
    std::vector<uint32_t> shards;
    std::vector<uint64_t> offsets;
    uint64_t n = 0;
    uint64_t ticket = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int status = RGL_OK;
    bool done = false;
    bool released = false;  // taken out of the ticket table by a completed wait
    uint32_t waiters = 0;   // threads inside rgl_server_wait on this request
    uint32_t batch_requests = 0;
    uint64_t batch_intervals = 0;
};

struct Worker {
    rgl_context* ctx = nullptr;
    DevBuf stage, dc, dbp, dp, dllr, dlp, dfl;
    StatsScratch sc;  // the stats stage's scratch (per worker: several batches run at once)
    uint32_t* h_counts = nullptr;
    uint64_t* h_bp = nullptr;
    double *h_p = nullptr, *h_llr = nullptr, *h_lp = nullptr;
    uint8_t* h_fl = nullptr;
    // the end of a batch: polled with yields, so that waiting workers leave their cores to the
    // callers and to each other, then waited on with a blocking synchronisation
    cudaEvent_t done = nullptr;
    std::thread th;
};

}  // namespace
}  // namespace rgl

using namespace rgl;

struct rgl_server {
    rgl_index* idx = nullptr;
    int device = 0;
    uint32_t D = 0;
    rgl_server_opts o{};
    bool with_bp = true;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> pending;
    uint64_t pending_n = 0;
    std::unordered_map<uint64_t, Req*> reqs;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::vector<std::unique_ptr<Worker>> workers;
    double worker_bytes = 0;
    uint64_t promised = 0;  // device bytes admitted batches will still allocate
    bool with_stats = false;
    std::vector<uint32_t> shard_chrom;
    // stats
    uint64_t memory_limited = 0, refused = 0, grown_bytes = 0;
    uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, intervals = 0, batch_req_sum = 0;
    std::vector<double> lat_ms;
    double first_submit = -1, last_done = 0;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// One batch on worker W: copies, pipeline, results.  Returns the batch status.
int run_batch(rgl_server* S, Worker* W, const std::vector<Req*>& batch) {
    rgl_context* c = W->ctx;
    cudaStream_t st = context_stream(c);
    const uint32_t R = (uint32_t)batch.size();
    std::vector<uint32_t> shards, rows;
    std::vector<uint64_t> off(1, 0);
    uint64_t at = 0;
    for (uint32_t j = 0; j < R; j++) {
        const Req* q = batch[j];
        if (q->n) {
            RGL_CUDA(cudaMemcpyAsync(W->stage.as<rgl_interval>() + at, q->r.intervals + q->offsets[0],
                                     q->n * sizeof(rgl_interval), cudaMemcpyHostToDevice, st));
        }
        for (size_t b = 0; b + 1 < q->offsets.size(); b++) {
            const uint64_t cnt = q->offsets[b + 1] - q->offsets[b];
            if (!cnt) continue;
            shards.push_back(q->shards[b]);
            rows.push_back(j);
            at += cnt;
            off.push_back(at);
        }
    }
    unsigned long long* d_bp = S->with_bp ? W->dbp.as<unsigned long long>() : nullptr;
    const size_t cells = (size_t)R * S->D;
    RGL_TRY(enqueue_block_rows(c, R, (uint32_t)shards.size(), shards.data(), rows.data(), off.data(),
                               W->stage.as<rgl_interval>(), &S->o.query, W->dc.as<uint32_t>(), d_bp));
    if (S->with_stats) {
        // the stats stage of the batch's rows: query length groups from the staged intervals,
        // FP64 p-values of every (row, source) cell (compute_analytic_pvalues,
        // src/tasks/query/pvalues.rs:22-77)
        rgl_batch b{R, (uint32_t)shards.size(), shards.data(), rows.data(), off.data(), W->stage.as<rgl_interval>()};
        RGL_TRY(batch_pvalues_enqueue(c, S->o.moments, &W->sc, &b, S->shard_chrom.data(),
                                      (uint32_t)S->shard_chrom.size(), S->o.bin_size, W->dc.as<uint32_t>(),
                                      W->dbp.as<uint64_t>(), W->dp.as<double>(), W->dllr.as<double>(),
                                      W->dlp.as<double>(), W->dfl.as<uint8_t>(), nullptr));
    }
    RGL_CUDA(cudaMemcpyAsync(W->h_counts, W->dc.p, cells * 4, cudaMemcpyDeviceToHost, st));
    if (d_bp) RGL_CUDA(cudaMemcpyAsync(W->h_bp, W->dbp.p, cells * 8, cudaMemcpyDeviceToHost, st));
    if (S->with_stats) {
        RGL_CUDA(cudaMemcpyAsync(W->h_p, W->dp.p, cells * 8, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(W->h_llr, W->dllr.p, cells * 8, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(W->h_lp, W->dlp.p, cells * 8, cudaMemcpyDeviceToHost, st));
        RGL_CUDA(cudaMemcpyAsync(W->h_fl, W->dfl.p, cells, cudaMemcpyDeviceToHost, st));
    }
    RGL_CUDA(cudaEventRecord(W->done, st));
    // wait by polling with yields (a blocking synchronisation's wake-up took up to ~30 ms on busy
    // hosts); a batch still running after 100 ms is waited for with the blocking call
    const auto w0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t q = cudaEventQuery(W->done);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) RGL_CUDA(q);
        if (std::chrono::steady_clock::now() - w0 > std::chrono::milliseconds(100)) {
            RGL_CUDA(cudaEventSynchronize(W->done));
            break;
        }
        std::this_thread::yield();
    }
    RGL_TRY(context_errors(c));
    const size_t D = S->D;
    for (uint32_t j = 0; j < R; j++) {
        const Req* q = batch[j];
        if (q->r.counts) std::memcpy(q->r.counts, W->h_counts + j * D, D * 4);
        if (q->r.overlap_bp) {
            if (d_bp) std::memcpy(q->r.overlap_bp, W->h_bp + j * D, D * 8);
            else std::memset(q->r.overlap_bp, 0, D * 8);
        }
        if (S->with_stats) {
            if (q->r.p_value) std::memcpy(q->r.p_value, W->h_p + j * D, D * 8);
            if (q->r.llr) std::memcpy(q->r.llr, W->h_llr + j * D, D * 8);
            if (q->r.log_p) std::memcpy(q->r.log_p, W->h_lp + j * D, D * 8);
            if (q->r.flags) std::memcpy(q->r.flags, W->h_fl + j * D, D);
        }
    }
    return RGL_OK;
}

uint64_t grow(const DevBuf& b, uint64_t bytes) { return bytes > b.cap ? bytes - b.cap : 0; }

// The stats stage's plan scratch for n intervals in nblk blocks (its tiles are at most
// n / kBlockSortCap + nblk): sort plan, order flags and run-head counts (StatsScratch::plan).
uint64_t stats_plan_bytes(uint64_t n, uint32_t nblk) {
    return (3ull * nblk + 2 * (n / kBlockSortCap + nblk) + 8) * 4;
}

// The stats stage's group offsets and block tables (StatsScratch::goff) for R rows and nblk blocks.
uint64_t stats_goff_bytes(rgl_server* S, uint32_t R, uint32_t nblk) {
    return (R + 1ull) * 8 + (nblk + 1ull) * 8 + (2ull * nblk + S->shard_chrom.size() + 1) * 4 + 64;
}

// Device bytes worker W would allocate to run a batch of n intervals in nblk blocks over R rows.
int batch_growth(rgl_server* S, Worker* W, uint64_t n, uint32_t R, uint32_t nblk, uint64_t* bytes) {
    uint64_t ws = 0;
    RGL_TRY(context_growth_bytes(W->ctx, n, 0, nblk, &ws));
    const uint64_t cells = (uint64_t)R * S->D;
    uint64_t b = ws + grow(W->stage, n * sizeof(rgl_interval)) + grow(W->dc, cells * 4 + 16) +
                 grow(W->dbp, cells * 8 + 16);
    if (S->with_stats) {
        b += grow(W->dp, cells * 8 + 16) + grow(W->dllr, cells * 8 + 16) + grow(W->dlp, cells * 8 + 16) +
             grow(W->dfl, cells + 16);
        // the stats stage's scratch: keys, lengths, runs and groups per interval (StatsScratch)
        b += grow(W->sc.key_a, n * 8 + 8) + grow(W->sc.key_b, n * 8 + 8) + grow(W->sc.len_a, n * 4 + 4) +
             grow(W->sc.len_b, n * 4 + 4) + grow(W->sc.ukey, n * 8 + 8) + grow(W->sc.agg, n * 32 + 32) +
             grow(W->sc.groups, n * 40 + 40) + grow(W->sc.plan, stats_plan_bytes(n, nblk)) +
             grow(W->sc.goff, stats_goff_bytes(S, R, nblk)) + grow(W->sc.runs, 64);
    }
    *bytes = b;
    return RGL_OK;
}

// Grows the worker's device buffers for a batch (the workspace grows inside the pipeline call).
int size_worker(rgl_server* S, Worker* W, uint64_t n, uint32_t R, uint32_t nblk) {
    const uint64_t cells = (uint64_t)R * S->D;
    RGL_TRY(W->stage.ensure(std::max<uint64_t>(n, 1) * sizeof(rgl_interval)));
    RGL_TRY(W->dc.ensure(cells * 4 + 16));
    RGL_TRY(W->dbp.ensure(cells * 8 + 16));
    if (S->with_stats) {
        RGL_TRY(W->dp.ensure(cells * 8 + 16));
        RGL_TRY(W->dllr.ensure(cells * 8 + 16));
        RGL_TRY(W->dlp.ensure(cells * 8 + 16));
        RGL_TRY(W->dfl.ensure(cells + 16));
        const uint64_t nn = std::max<uint64_t>(n, 1);
        RGL_TRY(W->sc.key_a.ensure(nn * 8 + 8));
        RGL_TRY(W->sc.key_b.ensure(nn * 8 + 8));
        RGL_TRY(W->sc.len_a.ensure(nn * 4 + 4));
        RGL_TRY(W->sc.len_b.ensure(nn * 4 + 4));
        RGL_TRY(W->sc.ukey.ensure(nn * 8 + 8));
        RGL_TRY(W->sc.agg.ensure(nn * 32 + 32));
        RGL_TRY(W->sc.groups.ensure(nn * 40 + 40));
        RGL_TRY(W->sc.plan.ensure(stats_plan_bytes(nn, nblk)));
        RGL_TRY(W->sc.goff.ensure(stats_goff_bytes(S, R, nblk)));
        RGL_TRY(W->sc.runs.ensure(64));
    }
    return RGL_OK;
}

uint64_t free_device_memory(rgl_server* S) {
    if (S->o.free_memory) return S->o.free_memory(S->o.free_memory_user);
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) return 0;
    return f;
}

void complete(rgl_server* S, const std::vector<Req*>& batch, const std::vector<int>& status, uint64_t n) {
    std::lock_guard<std::mutex> lk(S->mu);
    const double t = S->now();
    S->batches++;
    S->batch_req_sum += batch.size();
    for (size_t j = 0; j < batch.size(); j++) {
        Req* q = batch[j];
        q->status = status[j];
        q->t_done = t;
        q->done = true;
        q->batch_requests = (uint32_t)batch.size();
        q->batch_intervals = n;
        if (status[j] == RGL_OK) {
            S->completed++;
            S->intervals += q->n;
            S->lat_ms.push_back((t - q->t_submit) * 1e3);
        } else {
            S->failed++;
        }
        S->last_done = std::max(S->last_done, t);
    }
}

// Whether the batch the worker would form now (the oldest pending requests within
// max_batch_requests and batch_intervals) needs any device memory beyond what the worker holds;
// called with the server's lock held.  Growth is monotonic in the batch, so the whole tentative
// batch answers for each of its prefixes.
bool formation_grows(rgl_server* S, Worker* W) {
    uint64_t n = 0;
    uint32_t R = 0, nblk = 0;
    for (Req* q : S->pending) {
        if (R >= S->o.max_batch_requests || (R && n + q->n > S->o.batch_intervals)) break;
        n += q->n;
        nblk += (uint32_t)q->shards.size();
        R++;
    }
    uint64_t need = 0;
    return batch_growth(S, W, n, R, nblk, &need) != RGL_OK || need > 0;
}

void worker_main(rgl_server* S, Worker* W) {
    cudaSetDevice(S->device);
    std::vector<Req*> batch, refused;
    for (;;) {
        uint64_t n = 0, promise = 0;
        uint32_t nblk = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // admission needs the free device memory only when the batch would grow this worker's
            // buffers; the query (which can take milliseconds) runs without the lock, so that
            // submissions and the other workers do not wait on it
            uint64_t free_b = 0;
            bool have_free = false;
            for (;;) {
                S->cv_work.wait(lk, [&] { return S->stop || !S->pending.empty(); });
                if (S->pending.empty()) return;  // stop requested and the queue is drained
                if (have_free || !formation_grows(S, W)) break;
                lk.unlock();
                free_b = free_device_memory(S);
                have_free = true;
                lk.lock();
            }
            batch.clear();
            refused.clear();
            // what the device can still give this worker now (unbounded when nothing grows)
            const uint64_t keep = S->o.hbm_reserve_bytes + S->promised;
            const uint64_t avail = !have_free ? ~0ull : free_b > keep ? free_b - keep : 0;
            while (!S->pending.empty() && batch.size() < S->o.max_batch_requests) {
                Req* q = S->pending.front();
                if (!batch.empty() && n + q->n > S->o.batch_intervals) break;
                uint64_t need = 0;
                const uint32_t qb = (uint32_t)q->shards.size();
                if (batch_growth(S, W, n + q->n, (uint32_t)batch.size() + 1, nblk + qb, &need) != RGL_OK) need = ~0ull;
                if (need > 0 && !have_free) break;  // requests queued since the check: next round
                if (need > avail) {
                    if (!batch.empty()) {
                        S->memory_limited++;
                        break;
                    }
                    // not admissible even alone: fail it rather than wait for memory no one frees
                    S->pending.pop_front();
                    S->pending_n -= q->n;
                    refused.push_back(q);
                    continue;
                }
                promise = need;
                batch.push_back(q);
                n += q->n;
                nblk += qb;
                S->pending.pop_front();
            }
            S->pending_n -= n;
            S->promised += promise;
            const double t = S->now();
            for (Req* q : batch) q->t_start = t;
        }
        if (!refused.empty()) {
            std::lock_guard<std::mutex> lk(S->mu);
            const double t = S->now();
            for (Req* q : refused) {
                q->status = RGL_ERR_OOM;
                q->t_start = q->t_done = t;
                q->done = true;
                S->failed++;
                S->refused++;
            }
            S->cv_done.notify_all();
        }
        if (batch.empty()) continue;
        std::vector<int> status(batch.size(), RGL_OK);
        int s = size_worker(S, W, n, (uint32_t)batch.size(), nblk);
        if (s == RGL_OK) s = run_batch(S, W, batch);
        {
            std::lock_guard<std::mutex> lk(S->mu);  // the growth has happened: free memory shows it now
            S->promised -= promise;
            S->grown_bytes += promise;
        }
        if (s != RGL_OK && batch.size() > 1) {
            // isolate the failing request: every request of the batch again on its own
            std::vector<Req*> one(1);
            for (size_t j = 0; j < batch.size(); j++) {
                one[0] = batch[j];
                status[j] = run_batch(S, W, one);
            }
        } else if (s != RGL_OK) {
            status[0] = s;
        }
        complete(S, batch, status, n);
        S->cv_done.notify_all();
    }
}

void destroy_worker(Worker* W) {
    if (W->ctx) rgl_context_destroy(W->ctx);
    if (W->done) cudaEventDestroy(W->done);
    for (DevBuf* b : {&W->stage, &W->dc, &W->dbp, &W->dp, &W->dllr, &W->dlp, &W->dfl}) b->release();
    stats_scratch_release(&W->sc);
    for (void* h : {(void*)W->h_counts, (void*)W->h_bp, (void*)W->h_p, (void*)W->h_llr, (void*)W->h_lp, (void*)W->h_fl})
        if (h) cudaFreeHost(h);
}

int make_worker(rgl_server* S, Worker* W) {
    RGL_TRY(rgl_context_create(S->idx, nullptr, &W->ctx));
    RGL_CUDA(cudaEventCreateWithFlags(&W->done, cudaEventBlockingSync | cudaEventDisableTiming));
    const uint64_t cap = S->o.initial_intervals;
    const uint32_t R = S->o.max_batch_requests;
    // blocks per batch: at most one per (request, shard) for requests built from the shard list;
    // larger block tables grow the workspace on demand
    RGL_TRY(context_reserve_rows(W->ctx, cap, 0, R * std::max<uint32_t>(S->idx->num_shards, 1)));
    RGL_TRY(size_worker(S, W, cap, R, R * std::max<uint32_t>(S->idx->num_shards, 1)));
    const size_t cells = (size_t)R * S->D + 16;
    RGL_CUDA(cudaMallocHost(&W->h_counts, cells * 4));
    RGL_CUDA(cudaMallocHost(&W->h_bp, cells * 8));
    if (S->with_stats) {
        RGL_CUDA(cudaMallocHost(&W->h_p, cells * 8));
        RGL_CUDA(cudaMallocHost(&W->h_llr, cells * 8));
        RGL_CUDA(cudaMallocHost(&W->h_lp, cells * 8));
        RGL_CUDA(cudaMallocHost(&W->h_fl, cells));
    }
    return RGL_OK;
}

}  // namespace

extern "C" {

int rgl_server_create(rgl_index* index, const rgl_server_opts* opts, rgl_server** out) {
    clear_error();
    if (!index || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    auto S = std::make_unique<rgl_server>();
    S->idx = index;
    S->device = index->device;
    S->D = index->num_sources;
    S->t0 = std::chrono::steady_clock::now();
    if (opts) S->o = *opts;
    if (!S->o.workers) S->o.workers = 3;
    if (!S->o.max_batch_requests) S->o.max_batch_requests = 256;
    if (!S->o.batch_intervals) S->o.batch_intervals = 1ull << 23;
    if (!S->o.hbm_reserve_bytes) S->o.hbm_reserve_bytes = 4ull << 30;
    if (!S->o.max_pending_intervals) S->o.max_pending_intervals = 1ull << 28;
    S->o.batch_intervals = std::min<uint64_t>(S->o.batch_intervals, 200000000ull);  // one pipeline run
    // by default a worker reserves its whole workspace at creation: growing one later frees and
    // reallocates device buffers, which synchronises the device and stalls every other worker
    if (!S->o.initial_intervals) S->o.initial_intervals = S->o.batch_intervals;
    S->o.initial_intervals = std::min(S->o.initial_intervals, S->o.batch_intervals);
    if (!S->o.bin_size) S->o.bin_size = 100;
    S->with_bp = !(S->o.query.flags & RGL_QF_NO_OVERLAP);
    if (S->o.moments) {
        if (!S->with_bp) return fail(RGL_ERR_INVALID_ARGUMENT, "the stats stage needs the overlap (no RGL_QF_NO_OVERLAP)");
        if (S->o.num_shard_chrom && !S->o.shard_chrom) return fail(RGL_ERR_INVALID_ARGUMENT, "null shard_chrom");
        S->with_stats = true;
        S->shard_chrom.assign(S->o.shard_chrom, S->o.shard_chrom + S->o.num_shard_chrom);
        RGL_TRY(moments_prepare(S->o.moments));
    }
    RGL_CUDA(cudaSetDevice(S->device));
    // workers while free device memory (the provider's view) covers one more initial workspace
    for (uint32_t w = 0; w < S->o.workers; w++) {
        const uint64_t free0 = free_device_memory(S.get());
        if (w > 0 && (double)free0 < S->worker_bytes + (double)S->o.hbm_reserve_bytes) break;
        auto W = std::make_unique<Worker>();
        int s = make_worker(S.get(), W.get());
        if (s != RGL_OK) {
            destroy_worker(W.get());
            if (w == 0) {
                for (auto& x : S->workers) destroy_worker(x.get());
                return s;
            }
            clear_error();
            break;
        }
        const uint64_t free1 = free_device_memory(S.get());
        if (w == 0) S->worker_bytes = (double)(free0 > free1 ? free0 - free1 : 0);
        S->workers.push_back(std::move(W));
    }
    rgl_server* raw = S.release();
    for (auto& W : raw->workers) W->th = std::thread(worker_main, raw, W.get());
    *out = raw;
    return RGL_OK;
}

int rgl_server_submit(rgl_server* S, const rgl_request* req, uint64_t* ticket) {
    clear_error();
    if (!S || !req || !ticket) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    if (req->num_blocks && (!req->block_shards || !req->block_offsets || !req->intervals))
        return fail(RGL_ERR_INVALID_ARGUMENT, "incomplete request");
    auto q = std::make_unique<Req>();
    q->r = *req;
    q->shards.assign(req->block_shards, req->block_shards + req->num_blocks);
    q->offsets.assign(req->block_offsets, req->block_offsets + req->num_blocks + 1);
    if (!req->num_blocks) q->offsets.assign(1, 0);
    for (uint32_t b = 0; b < req->num_blocks; b++) {
        if (q->offsets[b + 1] < q->offsets[b]) return fail(RGL_ERR_INVALID_ARGUMENT, "block offsets must be non-decreasing");
        if (q->shards[b] >= S->idx->num_shards) return fail(RGL_ERR_INVALID_ARGUMENT, "shard id out of range");
    }
    q->n = q->offsets.back() - q->offsets.front();
    if (q->n > S->o.batch_intervals)
        return fail(RGL_ERR_INVALID_ARGUMENT, "request larger than the server's batch_intervals");
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return fail(RGL_ERR_INVALID_ARGUMENT, "server is stopping");
    if (S->pending_n + q->n > S->o.max_pending_intervals)
        return fail(RGL_ERR_OOM, "request queue full (max_pending_intervals)");
    q->ticket = S->next_ticket++;
    q->t_submit = S->now();
    if (S->first_submit < 0) S->first_submit = q->t_submit;
    S->submitted++;
    S->pending_n += q->n;
    *ticket = q->ticket;
    Req* raw = q.release();
    S->reqs[raw->ticket] = raw;
    S->pending.push_back(raw);
    S->cv_work.notify_one();
    return RGL_OK;
}

int rgl_server_wait(rgl_server* S, uint64_t ticket, uint32_t timeout_ms, rgl_request_info* info) {
    clear_error();
    if (!S) return fail(RGL_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(RGL_ERR_INVALID_ARGUMENT, "unknown ticket");
    Req* q = it->second;
    // Several threads may wait on one ticket: the request is freed only by the last of them to
    // leave, so no waiter reads it after the delete.
    q->waiters++;
    const bool done = S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->done; });
    q->waiters--;
    if (!done) return fail(RGL_ERR_TIMEOUT, "request not done yet");
    if (info) {
        info->status = q->status;
        info->batch_requests = q->batch_requests;
        info->batch_intervals = q->batch_intervals;
        info->intervals = q->n;
        info->submit_s = q->t_submit;
        info->start_s = q->t_start;
        info->done_s = q->t_done;
    }
    if (!q->released) {
        S->reqs.erase(q->ticket);
        q->released = true;
    }
    if (q->waiters == 0) delete q;
    return RGL_OK;
}

int rgl_server_get_stats(rgl_server* S, rgl_server_stats* out) {
    if (!S || !out) return fail(RGL_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = S->submitted;
    out->completed = S->completed;
    out->failed = S->failed;
    out->batches = S->batches;
    out->intervals = S->intervals;
    out->workers = (uint32_t)S->workers.size();
    out->pending = (uint32_t)S->pending.size();
    out->mean_batch_requests = S->batches ? (double)S->batch_req_sum / (double)S->batches : 0.0;
    out->first_submit_s = S->first_submit < 0 ? 0 : S->first_submit;
    out->last_done_s = S->last_done;
    out->worker_bytes = S->worker_bytes;
    out->memory_limited = S->memory_limited;
    out->refused = S->refused;
    out->grown_bytes = S->grown_bytes;
    if (!S->lat_ms.empty()) {
        std::vector<double> v(S->lat_ms);
        std::sort(v.begin(), v.end());
        // nearest-rank percentiles
        auto pct = [&](double p) {
            size_t k = (size_t)std::ceil(p / 100.0 * (double)v.size());
            return v[std::min(v.size(), std::max<size_t>(k, 1)) - 1];
        };
        out->p50_ms = pct(50);
        out->p99_ms = pct(99);
        out->p999_ms = pct(99.9);
        out->max_ms = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        out->mean_ms = sum / (double)v.size();
    }
    return RGL_OK;
}

int rgl_server_reset_stats(rgl_server* S) {
    if (!S) return fail(RGL_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    S->submitted = S->completed = S->failed = S->batches = S->intervals = S->batch_req_sum = 0;
    S->memory_limited = S->refused = 0;
    S->lat_ms.clear();
    S->first_submit = -1;
    S->last_done = 0;
    return RGL_OK;
}

int rgl_server_destroy(rgl_server* S) {
    clear_error();
    if (!S) return RGL_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto& W : S->workers)
        if (W->th.joinable()) W->th.join();
    cudaSetDevice(S->device);
    for (auto& W : S->workers) destroy_worker(W.get());
    for (auto& kv : S->reqs) delete kv.second;
    delete S;
    return RGL_OK;
}

}  // extern "C"
