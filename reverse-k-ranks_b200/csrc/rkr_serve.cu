// rkr_serve.cu -- a persistent serving loop over a resident index (rkr_server_*).
//
// The reference answers one query set per Retrieval call (src/app/ReverseRankIndex.cpp:191-192) with
// one topk; a server here keeps the index resident and answers a stream of requests, each a set of
// query items with a top-k per item, through continuous batching:
//   * requests wait in one FIFO queue; a worker takes requests from its head while they fit in a
//     batch: at most max_batch_queries query items, and at most the items whose per-batch work
//     arrays (2 bytes per (query, user) pair plus per-query state) fit the worker's memory budget;
//   * several workers run at once, each on its own CUDA stream with its own work arrays over the same
//     resident index data, so one batch's kernels overlap another's host steps and transfers;
//   * a worker pads its batch to the next of a few fixed sizes and replays the CUDA graph of the
//     batch's phase 1 captured for that size (both bound rounds: the fixed-shape part);
//   * each request is answered as a fresh index would answer it alone: QSRPNormalLP's carried
//     per-user scores (QSRPNormalLP.hpp:73,109,213-218) are scoped to the request (its own earlier
//     queries, then zero), so a request's result does not depend on what it was batched with.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {
namespace {

// Batch sizes a worker pads to (each has its own captured graph).
constexpr int kBuckets[] = {16, 32, 64, 128, 256, 512, 1024, 2048, 4096};
constexpr int kLastBucket = sizeof(kBuckets) / sizeof(kBuckets[0]) - 1;

struct Request {
    uint64_t ticket = 0;
    std::vector<float> query;      // [n][dim]
    std::vector<int32_t> k;        // [n]
    int32_t n = 0;
    int64_t n_out = 0;             // sum of k
    std::vector<rkr_user_rank> out;
    std::vector<rkr_query_stats> stats;
    int status = 1;                // 1 pending, RKR_OK done, < 0 failed
    char error[256] = "";
    double t_submit = 0, t_start = 0, t_done = 0;
};

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// A worker's view of the served index: the resident data is shared (read only), the stream, work
// arrays, graphs and profiler are its own.
rkr_index *shadow_create(const rkr_index *ix, int *status) {
    rkr_index *sh = new rkr_index(*ix);
    for (DevBuf *b : sh->workspaces()) {
        b->p = nullptr;
        b->bytes = 0;
    }
    sh->prof = Profiler();
    sh->graphs.clear();
    sh->graphs_on = true;
    sh->stream = nullptr;
    cudaError_t e = cudaSetDevice(sh->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sh->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        set_error("rkr_server_create: %s", cudaGetErrorString(e));
        *status = RKR_ERR_CUDA;
        delete sh;
        return nullptr;
    }
    *status = RKR_OK;
    return sh;
}

void shadow_destroy(rkr_index *sh) {
    if (!sh) return;
    cudaSetDevice(sh->device);
    if (sh->stream) cudaStreamSynchronize(sh->stream);
    for (DevBuf *b : sh->workspaces()) b->release();
    sh->prof.release();
    for (auto &g : sh->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (sh->stream) cudaStreamDestroy(sh->stream);
    // the shared resident buffers belong to the served index: forget them without freeing
    delete sh;
}

}  // namespace
}  // namespace rkr

using namespace rkr;

struct rkr_server {
    rkr_index *ix = nullptr;
    int method = 0, max_batch = 0, n_workers = 0;
    int64_t max_queries = 0;  // admission limit per batch (slots and memory)
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
    std::vector<std::thread> workers;
    std::vector<rkr_index *> shadows;
    bool stop = false;
    uint64_t next_ticket = 1;
    // counters
    int64_t n_batches = 0, n_requests = 0, n_queries = 0, n_padded = 0;
    double busy_s = 0;
};

namespace {

// One worker: take a batch, run it on the worker's stream, hand each request its rows.
void worker_loop(rkr_server *s, int w) {
    rkr_index *sh = s->shadows[w];
    cudaSetDevice(sh->device);
    const int dim = sh->dim;
    const int cap = s->max_batch <= kBuckets[kLastBucket] ? s->max_batch : kBuckets[kLastBucket];
    int bucket_max = kBuckets[kLastBucket];
    for (int b : kBuckets)
        if (b >= cap) { bucket_max = b; break; }
    // pinned staging and device buffers for the largest batch
    float *h_query = nullptr, *d_query = nullptr;
    rkr_user_rank *h_out = nullptr, *d_out = nullptr;
    rkr_query_stats *h_stats = nullptr, *d_stats = nullptr;
    int64_t out_cap = 0;  // result entries the staging holds (grown on demand)
    bool ok = cudaMallocHost(&h_query, sizeof(float) * (size_t) bucket_max * dim) == cudaSuccess &&
              cudaMalloc(&d_query, sizeof(float) * (size_t) bucket_max * dim) == cudaSuccess &&
              cudaMallocHost(&h_stats, sizeof(rkr_query_stats) * (size_t) bucket_max) == cudaSuccess &&
              cudaMalloc(&d_stats, sizeof(rkr_query_stats) * (size_t) bucket_max) == cudaSuccess;
    std::vector<int32_t> k(bucket_max), first(bucket_max);
    out_cap = (int64_t) bucket_max * 512;
    ok = ok && cudaMallocHost(&h_out, sizeof(rkr_user_rank) * (size_t) out_cap) == cudaSuccess &&
         cudaMalloc(&d_out, sizeof(rkr_user_rank) * (size_t) out_cap) == cudaSuccess;
    if (!ok) out_cap = 0;
    // warm-up, before the first request: every padded batch size the worker can form, from the largest
    // down, runs twice (the first run of the largest sizes the worker's work arrays, and a size's
    // first run is eager, its second captures the size's phase-1 graph), so that no request waits for
    // an allocation (which synchronises the device) or a capture
    if (ok) {
        for (int q = 0; q < bucket_max; q++)
            for (int j = 0; j < dim; j++) h_query[(size_t) q * dim + j] = (float) ((q + j) % 7) - 3.0f;
        bool warm = cudaMemcpyAsync(d_query, h_query, sizeof(float) * (size_t) bucket_max * dim,
                                    cudaMemcpyHostToDevice, sh->stream) == cudaSuccess;
        for (int bi = kLastBucket; warm && bi >= 0; bi--) {
            const int b = kBuckets[bi];
            if (b > bucket_max) continue;
            for (int q = 0; q < b; q++) {
                k[q] = 1;
                first[q] = q;
            }
            BatchSpec bs;
            bs.k = k.data();
            bs.req_first = first.data();
            for (int rep = 0; warm && rep < 2; rep++)
                warm = query_batch(sh, s->method, d_query, b, bs, d_out, d_stats, sh->stream) == RKR_OK;
        }
        cudaStreamSynchronize(sh->stream);  // a warm-up failure leaves the batches to size things themselves
    }
    for (;;) {
        std::vector<std::shared_ptr<Request>> batch;
        int nq = 0;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_work.wait(lock, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) break;  // stopping
            while (!s->queue.empty() && (batch.empty() || nq + s->queue.front()->n <= s->max_queries)) {
                batch.push_back(s->queue.front());
                nq += s->queue.front()->n;
                s->queue.pop_front();
            }
        }
        const double t0 = now_s();
        int rc = ok ? RKR_OK : RKR_ERR_NOMEM;
        if (!ok) set_error("rkr_server: worker buffers could not be allocated");
        int nb = nq;
        for (int b : kBuckets)
            if (b >= nq) { nb = b; break; }
        if (rc == RKR_OK) {
            // pack the requests, then pad with one-query requests of k = 1 (their rows are dropped)
            int at = 0;
            for (auto &r : batch) {
                r->t_start = t0;
                std::memcpy(h_query + (size_t) at * dim, r->query.data(), sizeof(float) * (size_t) r->n * dim);
                for (int i = 0; i < r->n; i++) {
                    k[at + i] = r->k[i];
                    first[at + i] = at;
                }
                at += r->n;
            }
            for (int q = nq; q < nb; q++) {
                std::memcpy(h_query + (size_t) q * dim, h_query, sizeof(float) * dim);
                k[q] = 1;
                first[q] = q;
            }
            int64_t n_out = 0;
            for (int q = 0; q < nb; q++) n_out += k[q];
            cudaError_t e = cudaSuccess;
            if (n_out > out_cap) {
                cudaFreeHost(h_out);
                cudaFree(d_out);
                h_out = nullptr;
                d_out = nullptr;
                out_cap = std::max<int64_t>(n_out, (int64_t) bucket_max * 128);
                e = cudaMallocHost(&h_out, sizeof(rkr_user_rank) * (size_t) out_cap);
                if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(rkr_user_rank) * (size_t) out_cap);
                if (e != cudaSuccess) out_cap = 0;
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_query, h_query, sizeof(float) * (size_t) nb * dim, cudaMemcpyHostToDevice,
                                            sh->stream);
            if (e != cudaSuccess) {
                set_error("rkr_server: %s", cudaGetErrorString(e));
                rc = RKR_ERR_CUDA;
            }
            if (rc == RKR_OK) {
                BatchSpec bs;
                bs.k = k.data();
                bs.req_first = first.data();
                rc = query_batch(sh, s->method, d_query, nb, bs, d_out, d_stats, sh->stream);
            }
            if (rc == RKR_OK) {
                e = cudaMemcpyAsync(h_out, d_out, sizeof(rkr_user_rank) * (size_t) n_out, cudaMemcpyDeviceToHost,
                                    sh->stream);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(h_stats, d_stats, sizeof(rkr_query_stats) * (size_t) nb, cudaMemcpyDeviceToHost,
                                        sh->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(sh->stream);
                if (e != cudaSuccess) {
                    set_error("rkr_server: %s", cudaGetErrorString(e));
                    rc = RKR_ERR_CUDA;
                }
            }
        }
        const double t1 = now_s();
        {
            std::lock_guard<std::mutex> lock(s->mu);
            int64_t at_out = 0;
            int at = 0;
            for (auto &r : batch) {
                if (rc == RKR_OK) {
                    r->out.assign(h_out + at_out, h_out + at_out + r->n_out);
                    r->stats.assign(h_stats + at, h_stats + at + r->n);
                    r->status = RKR_OK;
                } else {
                    r->status = rc;
                    std::strncpy(r->error, rkr_last_error(), sizeof(r->error) - 1);
                }
                r->t_done = t1;
                at_out += r->n_out;
                at += r->n;
            }
            s->n_batches++;
            s->n_requests += (int64_t) batch.size();
            s->n_queries += nq;
            s->n_padded += nb - nq;
            s->busy_s += t1 - t0;
        }
        s->cv_done.notify_all();
    }
    cudaFreeHost(h_query);
    cudaFree(d_query);
    cudaFreeHost(h_out);
    cudaFree(d_out);
    cudaFreeHost(h_stats);
    cudaFree(d_stats);
}

}  // namespace

extern "C" {

int rkr_server_create(rkr_index *ix, const rkr_server_config *cfg, rkr_server **out) {
    RKR_REQUIRE(ix && cfg && out, "null argument");
    *out = nullptr;
    if (ix->sharded()) {
        set_error("rkr_server_create: the index is a user shard");
        return RKR_ERR_STATE;
    }
    RKR_REQUIRE(cfg->method == RKR_METHOD_QS || cfg->method == RKR_METHOD_QSRP_NORMAL_LP,
                "rkr_server_create: method %d (QS or QSRPNormalLP; US answers fixed sets of 100 queries)", cfg->method);
    RKR_REQUIRE(cfg->max_batch_queries >= 1 && cfg->max_batch_queries <= kMaxChunkQueries,
                "rkr_server_create: max_batch_queries %d outside [1, %d]", cfg->max_batch_queries, kMaxChunkQueries);
    RKR_REQUIRE(cfg->n_workers >= 1 && cfg->n_workers <= 8, "rkr_server_create: n_workers %d outside [1, 8]",
                cfg->n_workers);
    RKR_REQUIRE(cfg->workspace_bytes >= 0, "rkr_server_create: negative workspace_bytes");
    // the method's structures must be loaded; one warm-up query through the index builds every
    // lazily built shared structure (the pair scores' digit tiles) and the refinement's item tiles
    // are built here, before the workers share the index read-only
    {
        int32_t na = 0;
        RKR_TRY(ensure_device(ix));
        std::vector<float> q(ix->dim, 0.0f);
        for (int j = 0; j < ix->dim; j++) q[j] = (float) (j % 7) - 3.0f;
        std::vector<rkr_user_rank> o(1);
        RKR_TRY(rkr_retrieval(ix, cfg->method, q.data(), 1, 1, o.data(), nullptr, &na));
        RKR_TRY(refine_tc_tiles(ix, true, ix->stream));
        RKR_CUDA(cudaStreamSynchronize(ix->stream));
    }
    rkr_server *s = new rkr_server();
    s->ix = ix;
    s->method = cfg->method;
    s->max_batch = cfg->max_batch_queries;
    s->n_workers = cfg->n_workers;
    // admission by memory: a query's per-batch work arrays are about 2 bytes per user plus its
    // threshold buckets and candidate rows
    const int64_t per_query = ix->n_user * 2 + (int64_t) (ix->n_sample + 1) * 8 + 64 * 1024;
    const int64_t by_mem = cfg->workspace_bytes > 0 ? std::max<int64_t>(1, cfg->workspace_bytes / per_query)
                                                    : (int64_t) kMaxChunkQueries;
    s->max_queries = std::min<int64_t>(s->max_batch, by_mem);
    for (int w = 0; w < s->n_workers; w++) {
        int st = RKR_OK;
        rkr_index *sh = shadow_create(ix, &st);
        if (!sh) {
            for (rkr_index *x : s->shadows) shadow_destroy(x);
            delete s;
            return st;
        }
        s->shadows.push_back(sh);
    }
    for (int w = 0; w < s->n_workers; w++) s->workers.emplace_back(worker_loop, s, w);
    *out = s;
    return RKR_OK;
}

int rkr_server_submit(rkr_server *s, const float *query, int32_t n_query, const int32_t *k_per_q, uint64_t *ticket) {
    RKR_REQUIRE(s && query && k_per_q && ticket, "null argument");
    RKR_REQUIRE(n_query >= 1 && n_query <= s->max_queries,
                "rkr_server_submit: %d query items outside [1, %lld] (the server's batch limit)", n_query,
                (long long) s->max_queries);
    auto r = std::make_shared<Request>();
    r->n = n_query;
    r->query.assign(query, query + (size_t) n_query * s->ix->dim);
    r->k.assign(k_per_q, k_per_q + n_query);
    for (int i = 0; i < n_query; i++) {
        RKR_REQUIRE(r->k[i] >= 1 && r->k[i] <= s->ix->n_user && r->k[i] <= 4096, "rkr_server_submit: k[%d] = %d",
                    i, r->k[i]);
        r->n_out += r->k[i];
    }
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        RKR_REQUIRE(!s->stop, "rkr_server_submit: the server is stopping");
        r->ticket = s->next_ticket++;
        s->live[r->ticket] = r;
        s->queue.push_back(r);
    }
    s->cv_work.notify_one();
    *ticket = r->ticket;
    return RKR_OK;
}

int rkr_server_wait(rkr_server *s, uint64_t ticket, double timeout_s, rkr_user_rank *out, rkr_query_stats *stats,
                    double *latency_s) {
    RKR_REQUIRE(s, "null server");
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        auto it = s->live.find(ticket);
        RKR_REQUIRE(it != s->live.end(), "rkr_server_wait: unknown ticket %llu", (unsigned long long) ticket);
        r = it->second;
        const auto pred = [&] { return r->status != 1; };
        if (timeout_s < 0) {
            s->cv_done.wait(lock, pred);
        } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), pred)) {
            set_error("rkr_server_wait: ticket %llu not done within %.3f s", (unsigned long long) ticket, timeout_s);
            return RKR_ERR_STATE;
        }
        s->live.erase(ticket);
    }
    if (r->status != RKR_OK) {
        set_error("%s", r->error);
        return r->status;
    }
    if (out) std::memcpy(out, r->out.data(), sizeof(rkr_user_rank) * (size_t) r->n_out);
    if (stats) std::memcpy(stats, r->stats.data(), sizeof(rkr_query_stats) * (size_t) r->n);
    if (latency_s) {
        latency_s[0] = r->t_done - r->t_submit;
        latency_s[1] = r->t_start - r->t_submit;
    }
    return RKR_OK;
}

int rkr_server_counters(rkr_server *s, int64_t *batches, int64_t *requests, int64_t *queries, int64_t *padded,
                        double *busy_s) {
    RKR_REQUIRE(s, "null server");
    std::lock_guard<std::mutex> lock(s->mu);
    if (batches) *batches = s->n_batches;
    if (requests) *requests = s->n_requests;
    if (queries) *queries = s->n_queries;
    if (padded) *padded = s->n_padded;
    if (busy_s) *busy_s = s->busy_s;
    return RKR_OK;
}

int rkr_server_destroy(rkr_server *s) {
    if (!s) return RKR_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    for (rkr_index *sh : s->shadows) shadow_destroy(sh);
    delete s;
    return RKR_OK;
}

}  // extern "C"
