// User shards: the count exchange of a sharded query, the in-process exchange group, and the host
// merge of the shards' partial rows.
//
// A sharded query runs the whole pipeline on every shard.  Each selection of the pipeline reads a
// per-query count array (coarse and exact regression levels, threshold groups and buckets, the
// round-1 class counts) and takes a k-th smallest value or a class count from it; summed over the
// shards, those arrays are the unsharded index's, so every shard makes the same decisions, and then
// classifies, refines and assembles its own users.  This replaces the all-gather of each shard's k
// smallest bounds that PruneCandidateByBound's global step would need with a fixed-size sum of
// small arrays (the reference's PruneCandidateByBound.hpp:19-179 holds every user in one process).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {

__global__ void shard_axpy_kernel(int32_t *__restrict__ c, const int32_t *__restrict__ snap, int64_t n, int sign) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        c[i] += sign * snap[i];
}

__global__ void shard_local_counts_kernel(const int2 *__restrict__ cnt, int nchunks, int nq, int keep_base,
                                          QueryCounts *__restrict__ counts) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    int64_t c = 0;
    for (int i = 0; i < nchunks; i++) c += cnt[(int64_t) q * nchunks + i].y;
    counts[q].n_cand = (int32_t) c;
    if (!keep_base) counts[q].ip_base = 0;
}

int shard_sum(rkr_index *ix, int32_t *counts, int64_t n, cudaStream_t st) {
    if (!ix->sharded() || n <= 0) return RKR_OK;
    const int rc = ix->shard.fn(ix->shard.ctx, counts, n, (void *) st);
    if (rc != 0) {
        set_error("user shard %d: the count exchange failed (%d)", ix->shard.index, rc);
        return RKR_ERR_STATE;
    }
    return RKR_OK;
}

int shard_snapshot(rkr_index *ix, int slot, const int32_t *counts, int64_t n, cudaStream_t st) {
    if (!ix->sharded() || n <= 0) return RKR_OK;
    RKR_TRY(ix->ws_snap[slot].ensure(sizeof(int32_t) * (size_t) n));
    RKR_CUDA(cudaMemcpyAsync(ix->ws_snap[slot].p, counts, sizeof(int32_t) * (size_t) n, cudaMemcpyDeviceToDevice, st));
    return RKR_OK;
}

int shard_sum_delta(rkr_index *ix, int slot, int32_t *counts, int64_t n, cudaStream_t st) {
    if (!ix->sharded() || n <= 0) return RKR_OK;
    const int32_t *snap = ix->ws_snap[slot].as<int32_t>();
    const unsigned g = (unsigned) std::min<int64_t>(148 * 8, (n + 255) / 256);
    shard_axpy_kernel<<<g, 256, 0, st>>>(counts, snap, n, -1);  // this shard's additions
    RKR_CUDA(cudaGetLastError());
    RKR_TRY(shard_sum(ix, counts, n, st));
    shard_axpy_kernel<<<g, 256, 0, st>>>(counts, snap, n, 1);
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

int shard_sum_host(rkr_index *ix, int32_t v, int32_t *sum, cudaStream_t st) {
    *sum = v;
    if (!ix->sharded()) return RKR_OK;
    RKR_TRY(ix->ws_shard.ensure(sizeof(int32_t)));
    int32_t *d = ix->ws_shard.as<int32_t>();
    RKR_CUDA(cudaMemcpyAsync(d, &v, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    RKR_TRY(shard_sum(ix, d, 1, st));
    RKR_CUDA(cudaMemcpyAsync(sum, d, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    return RKR_OK;
}

}  // namespace rkr

namespace {

// The in-process exchange: a generation-counted barrier with the running sum.  A member that
// waits past the timeout marks the group broken, and every later call fails at once.
struct HostExchange {
    int n_members = 0;
    double timeout_s = 0;
    std::mutex mu;
    std::condition_variable cv;
    int arrived = 0;
    uint64_t generation = 0;
    int64_t n_elems = 0;
    std::vector<int64_t> acc, result;
    bool broken = false;
};

}  // namespace

using rkr::set_error;

extern "C" {

int rkr_host_exchange_create(int32_t n_members, double timeout_s, void **group) {
    RKR_REQUIRE(group, "null group pointer");
    RKR_REQUIRE(n_members >= 1 && n_members <= 1024, "n_members %d outside [1, 1024]", n_members);
    RKR_REQUIRE(timeout_s > 0, "timeout_s must be positive");
    auto *g = new (std::nothrow) HostExchange();
    if (!g) {
        set_error("host exchange: out of memory");
        return RKR_ERR_NOMEM;
    }
    g->n_members = n_members;
    g->timeout_s = timeout_s;
    *group = g;
    return RKR_OK;
}

int rkr_host_exchange_destroy(void *group) {
    delete static_cast<HostExchange *>(group);
    return RKR_OK;
}

int rkr_host_exchange(void *group, int32_t *counts, int64_t n, void *stream) {
    auto *g = static_cast<HostExchange *>(group);
    if (!g || !counts || n < 0) return RKR_ERR_INVALID;
    cudaStream_t st = (cudaStream_t) stream;
    std::vector<int32_t> mine((size_t) n);
    if (stream) {
        if (cudaMemcpyAsync(mine.data(), counts, sizeof(int32_t) * (size_t) n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return RKR_ERR_CUDA;
    } else {
        std::memcpy(mine.data(), counts, sizeof(int32_t) * (size_t) n);
    }
    std::vector<int64_t> sum;
    {
        std::unique_lock<std::mutex> lk(g->mu);
        if (g->broken) return RKR_ERR_STATE;
        if (g->arrived == 0) {
            g->n_elems = n;
            g->acc.assign((size_t) n, 0);
        } else if (g->n_elems != n) {
            g->broken = true;  // the members disagree on the call sequence
            g->cv.notify_all();
            return RKR_ERR_STATE;
        }
        for (int64_t i = 0; i < n; i++) g->acc[(size_t) i] += mine[(size_t) i];
        const uint64_t gen = g->generation;
        if (++g->arrived == g->n_members) {
            g->result.swap(g->acc);
            g->arrived = 0;
            g->generation++;
            g->cv.notify_all();
        } else {
            const auto limit = std::chrono::duration<double>(g->timeout_s);
            if (!g->cv.wait_for(lk, limit, [&] { return g->generation != gen || g->broken; }) || g->broken) {
                g->broken = true;
                g->cv.notify_all();
                return RKR_ERR_STATE;
            }
        }
        // the next generation cannot complete before this member joins it, so result is this one's
        sum = g->result;
    }
    for (int64_t i = 0; i < n; i++) mine[(size_t) i] = (int32_t) sum[(size_t) i];
    if (stream) {
        if (cudaMemcpyAsync(counts, mine.data(), sizeof(int32_t) * (size_t) n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return RKR_ERR_CUDA;
    } else {
        std::memcpy(counts, mine.data(), sizeof(int32_t) * (size_t) n);
    }
    return RKR_OK;
}

// The reference's assembly (QSRPNormalLP.hpp:213-226, QS.hpp:185-198) over the shards' parts: the
// result users in user-id order (shard order is user order, and each part lists its results by
// user id), then the candidates by (rank, user id), merged from the parts' sorted runs.
int rkr_shard_merge(int32_t n_shards, int32_t n_query, const int32_t *k_per_q, const rkr_user_rank *const *parts,
                    const int32_t *const *n_fronts, const rkr_query_stats *const *stats, rkr_user_rank *out,
                    rkr_query_stats *stats_out) {
    RKR_REQUIRE(n_shards >= 1 && n_query >= 0, "bad shard or query count");
    RKR_REQUIRE(k_per_q && parts && n_fronts && out, "null argument");
    for (int s = 0; s < n_shards; s++) RKR_REQUIRE(parts[s] && n_fronts[s], "null part of shard %d", s);
    RKR_REQUIRE(!stats_out || stats, "stats_out needs the shards' stats");
    if (stats)
        for (int s = 0; s < n_shards; s++) RKR_REQUIRE(stats[s], "null stats of shard %d", s);
    int64_t at = 0;
    std::vector<int> pos((size_t) n_shards), end((size_t) n_shards);
    for (int q = 0; q < n_query; q++) {
        const int k = k_per_q[q];
        RKR_REQUIRE(k >= 1, "k_per_q[%d] = %d", q, k);
        rkr_user_rank *o = out + at;
        int filled = 0;
        for (int s = 0; s < n_shards && filled < k; s++) {
            const int nf = n_fronts[s][q];
            RKR_REQUIRE(nf >= 0 && nf <= k, "n_fronts[%d][%d] = %d outside [0, %d]", s, q, nf, k);
            for (int i = 0; i < nf && filled < k; i++) o[filled++] = parts[s][at + i];
        }
        for (int s = 0; s < n_shards; s++) {
            pos[(size_t) s] = n_fronts[s][q];
            int e = pos[(size_t) s];
            while (e < k && parts[s][at + e].user_id >= 0) e++;
            end[(size_t) s] = e;
        }
        while (filled < k) {
            int best = -1;
            for (int s = 0; s < n_shards; s++) {
                if (pos[(size_t) s] >= end[(size_t) s]) continue;
                const rkr_user_rank &c = parts[s][at + pos[(size_t) s]];
                if (best < 0) { best = s; continue; }
                const rkr_user_rank &b = parts[best][at + pos[(size_t) best]];
                if (c.rank < b.rank || (c.rank == b.rank && c.user_id < b.user_id)) best = s;
            }
            if (best < 0) break;
            o[filled++] = parts[best][at + pos[(size_t) best]++];
        }
        for (; filled < k; filled++) o[filled] = rkr_user_rank{-1, -1, -1.0f};
        if (stats_out) {
            rkr_query_stats t = stats[0][q];  // n_prune and n_result are every shard's
            for (int s = 1; s < n_shards; s++) {
                t.n_refine += stats[s][q].n_refine;
                t.n_candidate += stats[s][q].n_candidate;
                t.n_compute_item += stats[s][q].n_compute_item;
                t.ip_cost += stats[s][q].ip_cost;
            }
            stats_out[q] = t;
        }
        at += k;
    }
    return RKR_OK;
}

}  // extern "C"
