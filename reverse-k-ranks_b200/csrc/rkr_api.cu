// rkr_api.cu -- the C ABI of librkr_b200.so (declared in include/rkr.h).
#include <algorithm>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int ensure_device(const rkr_index *ix) {
    RKR_CUDA(cudaSetDevice(ix->device));
    return RKR_OK;
}

// ||v|| = sqrt(InnerProduct(v + off, v + off, len)) per row (RefineCPUIPBound.hpp:433-437,
// RefineCPUPartDimPartNorm.hpp:39-54, PartDimPartNorm.hpp:41-50).
__global__ void row_norm_kernel(const float *__restrict__ v, int64_t n, int dim, int off, float *__restrict__ out) {
    const int64_t r = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float *p = v + r * dim + off;
    out[r] = __fsqrt_rn(exact_dot(p, p, dim - off));
}

// Per user, the last (smallest) threshold of each group of thr_group(S) consecutive thresholds;
// unused slots hold -inf.
__global__ void thr_summary_kernel(const float *__restrict__ thr, int64_t n_user, int S, float *__restrict__ summ) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_user * ThrSummary::kMaxGroups) return;
    const int64_t u = i / ThrSummary::kMaxGroups;
    const int j = (int) (i % ThrSummary::kMaxGroups);
    const int g = thr_group(S), nb = (S + g - 1) / g;
    summ[i] = j < nb ? thr[u * S + min(g * j + g - 1, S - 1)] : -INFINITY;
}

__global__ void gather_rows_kernel(const float *__restrict__ src, const int32_t *__restrict__ idx, int64_t n, int dim,
                                   float *__restrict__ dst) {
    const int64_t r = blockIdx.x;
    if (r >= n) return;
    const float *s = src + (int64_t) idx[r] * dim;
    for (int j = threadIdx.x; j < dim; j += blockDim.x) dst[r * dim + j] = s[j];
}

__global__ void to_kmajor_kernel(const float *__restrict__ src, const int32_t *__restrict__ idx, int64_t n, int dim,
                                 int64_t ld, float *__restrict__ dst) {
    __shared__ float t[32][33];
    const int64_t r0 = (int64_t) blockIdx.x * 32;
    const int d0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int64_t r = r0 + i;
        const int d = d0 + threadIdx.x;
        t[i][threadIdx.x] = r < n && d < dim ? src[(idx ? (int64_t) idx[r] : r) * dim + d] : 0.0f;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int d = d0 + i;
        const int64_t r = r0 + threadIdx.x;
        if (d < dim && r < ld) dst[(int64_t) d * ld + r] = t[threadIdx.x][i];
    }
}

int to_kmajor(const float *src, const int32_t *idx, int64_t n, int dim, float *dst, cudaStream_t st) {
    const int64_t ld = kmajor_ld(n);
    if (ld == 0) return RKR_OK;
    dim3 grid((unsigned) (ld / 32), (unsigned) ((dim + 31) / 32));
    to_kmajor_kernel<<<grid, dim3(32, 8), 0, st>>>(src, idx, n, dim, ld, dst);
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

// Norms the refinement bound needs for the current check_dim (recomputed when it changes).
int refine_prepare_norms(rkr_index *ix) {
    const int c = ix->check_dim;
    RKR_TRY(ix->item_rnorm.ensure(sizeof(float) * ix->n_item));
    RKR_TRY(ix->user_rnorm.ensure(sizeof(float) * ix->n_user));
    row_norm_kernel<<<(unsigned) ((ix->n_item + 255) / 256), 256, 0, ix->stream>>>(ix->item_sorted.as<float>(), ix->n_item,
                                                                                  ix->dim, c, ix->item_rnorm.as<float>());
    RKR_CUDA(cudaGetLastError());
    row_norm_kernel<<<(unsigned) ((ix->n_user + 255) / 256), 256, 0, ix->stream>>>(ix->user.as<float>(), ix->n_user,
                                                                                  ix->dim, c, ix->user_rnorm.as<float>());
    RKR_CUDA(cudaGetLastError());
    if (ix->has_svd) {
        RKR_TRY(ix->svd_unorm.ensure(sizeof(float) * ix->n_user));
        row_norm_kernel<<<(unsigned) ((ix->n_user + 255) / 256), 256, 0, ix->stream>>>(
            ix->svd_user.as<float>(), ix->n_user, ix->dim, c, ix->svd_unorm.as<float>());
        RKR_CUDA(cudaGetLastError());
    }
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

// Group summaries of the current thresholds (enqueued on the index stream).
int thr_summary_build(rkr_index *ix) {
    const int64_t n = ix->n_user * ThrSummary::kMaxGroups;
    RKR_TRY(ix->thr_summ.ensure(sizeof(float) * (size_t) n));
    thr_summary_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, ix->stream>>>(ix->thr.as<float>(), ix->n_user,
                                                                            ix->n_sample, ix->thr_summ.as<float>());
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

}  // namespace rkr

using namespace rkr;

extern "C" {

const char *rkr_last_error(void) { return g_err; }

int rkr_version(void) { return 1; }

int rkr_index_create(int32_t device, const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t dim,
                     rkr_index **out) {
    RKR_REQUIRE(out && user && item, "rkr_index_create: null argument");
    RKR_REQUIRE(n_user > 0 && n_item > 0 && dim > 0, "rkr_index_create: empty user/item set or dim");
    RKR_REQUIRE(n_user < (int64_t(1) << 31) && n_item < (int64_t(1) << 31) && dim <= 4096,
                "rkr_index_create: sizes out of range");
    *out = nullptr;
    int n_dev = 0;
    RKR_CUDA(cudaGetDeviceCount(&n_dev));
    RKR_REQUIRE(device >= 0 && device < n_dev, "rkr_index_create: device %d of %d", device, n_dev);
    rkr_index *ix = new rkr_index();
    ix->device = device;
    // RKR_REFINE_TC=0 keeps refinement on the exact tiles (both paths give the same results)
    if (const char *v = getenv("RKR_REFINE_TC")) ix->refine_tc_on = strcmp(v, "0") != 0;
    // RKR_SCORES_TC=0 keeps the bound rounds' pair scores on the exact tiles (same results)
    if (const char *v = getenv("RKR_SCORES_TC")) ix->scores_tc_on = strcmp(v, "0") != 0;
    // RKR_COMPACT_SPARSE=0 gives every query the two-pass ordered compaction (same results)
    if (const char *v = getenv("RKR_COMPACT_SPARSE")) ix->compact_sparse_on = strcmp(v, "0") != 0;
    ix->n_user = n_user;
    ix->n_item = n_item;
    ix->dim = dim;
    auto fail = [&](int s) {
        rkr_index_destroy(ix);
        return s;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ix->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        set_error("rkr_index_create: %s", cudaGetErrorString(e));
        return fail(RKR_ERR_CUDA);
    }
    int s;
    if ((s = ix->user.ensure(sizeof(float) * n_user * dim)) || (s = ix->item.ensure(sizeof(float) * n_item * dim)) ||
        (s = ix->item_sorted.ensure(sizeof(float) * n_item * dim)) || (s = ix->item_norm.ensure(sizeof(float) * n_item)) ||
        (s = ix->qip_state.ensure(sizeof(float) * n_user)))
        return fail(s);
    e = cudaMemcpyAsync(ix->user.p, user, sizeof(float) * n_user * dim, cudaMemcpyHostToDevice, ix->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ix->item.p, item, sizeof(float) * n_item * dim, cudaMemcpyHostToDevice, ix->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ix->qip_state.p, 0, sizeof(float) * n_user, ix->stream);
    if (e != cudaSuccess) {
        set_error("rkr_index_create: upload: %s", cudaGetErrorString(e));
        return fail(RKR_ERR_CUDA);
    }
    // Items by norm, descending (RefineCPUIPBound.hpp:430-452).
    row_norm_kernel<<<(unsigned) ((n_item + 255) / 256), 256, 0, ix->stream>>>(ix->item.as<float>(), n_item, dim, 0,
                                                                              ix->item_norm.as<float>());
    std::vector<float> norm(n_item);
    e = cudaMemcpyAsync(norm.data(), ix->item_norm.p, sizeof(float) * n_item, cudaMemcpyDeviceToHost, ix->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ix->stream);
    if (e != cudaSuccess) {
        set_error("rkr_index_create: norms: %s", cudaGetErrorString(e));
        return fail(RKR_ERR_CUDA);
    }
    std::vector<int32_t> order(n_item);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return norm[a] > norm[b]; });
    ix->h_item_order = order;
    ix->h_item_norm_sorted.resize(n_item);
    for (int64_t i = 0; i < n_item; i++) ix->h_item_norm_sorted[i] = norm[order[i]];
    if ((s = ix->ws_misc.ensure(sizeof(int32_t) * n_item))) return fail(s);
    e = cudaMemcpyAsync(ix->ws_misc.p, order.data(), sizeof(int32_t) * n_item, cudaMemcpyHostToDevice, ix->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ix->item_norm.p, ix->h_item_norm_sorted.data(), sizeof(float) * n_item, cudaMemcpyHostToDevice,
                            ix->stream);
    if (e != cudaSuccess) {
        set_error("rkr_index_create: %s", cudaGetErrorString(e));
        return fail(RKR_ERR_CUDA);
    }
    gather_rows_kernel<<<(unsigned) n_item, 64, 0, ix->stream>>>(ix->item.as<float>(), ix->ws_misc.as<int32_t>(), n_item,
                                                                dim, ix->item_sorted.as<float>());
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("rkr_index_create: %s", cudaGetErrorString(e));
        return fail(RKR_ERR_CUDA);
    }
    // k-major copies for the refinement tiles
    const size_t km = sizeof(float) * (size_t) dim * (size_t) kmajor_ld(n_item);
    const size_t kmu = sizeof(float) * (size_t) dim * (size_t) kmajor_ld(n_user);
    if ((s = ix->user_km.ensure(kmu)) ||
        (s = to_kmajor(ix->user.as<float>(), nullptr, n_user, dim, ix->user_km.as<float>(), ix->stream)))
        return fail(s);
    if ((s = ix->item_km.ensure(km)) || (s = ix->item_sorted_km.ensure(km)) ||
        (s = to_kmajor(ix->item.as<float>(), nullptr, n_item, dim, ix->item_km.as<float>(), ix->stream)) ||
        (s = to_kmajor(ix->item_sorted.as<float>(), nullptr, n_item, dim, ix->item_sorted_km.as<float>(), ix->stream)))
        return fail(s);
    e = cudaStreamSynchronize(ix->stream);
    if (e != cudaSuccess) {
        set_error("rkr_index_create: %s", cudaGetErrorString(e));
        return fail(RKR_ERR_CUDA);
    }
    *out = ix;
    return RKR_OK;
}

int rkr_index_destroy(rkr_index *ix) {
    if (!ix) return RKR_OK;
    cudaSetDevice(ix->device);
    if (ix->stream) cudaStreamSynchronize(ix->stream);
    for (DevBuf *b : {&ix->user, &ix->item, &ix->item_sorted, &ix->item_norm, &ix->item_rnorm, &ix->user_rnorm,
                      &ix->sample_rank, &ix->thr, &ix->thr_summ, &ix->reg_rank, &ix->reg, &ix->lvt, &ix->transfer_item,
                      &ix->svd_user, &ix->svd_user_km, &ix->user_km, &ix->item_km, &ix->item_sorted_km, &ix->ri_item_split,
                      &ix->ri_imeta_split, &ix->ri_item_full, &ix->ri_imeta_full, &ix->svd_unorm, &ix->qip_state,
                      &ix->sc_user_split, &ix->sc_umeta_split, &ix->sc_user_full, &ix->sc_umeta_full, &ix->sc_cdf_tab})
        b->release();
    for (DevBuf *b : ix->workspaces()) b->release();
    ix->prof.release();
    for (auto &g : ix->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (ix->stream) cudaStreamDestroy(ix->stream);
    delete ix;
    return RKR_OK;
}

int rkr_index_set_check_dim(rkr_index *ix, int32_t check_dim) {
    RKR_REQUIRE(ix, "null index");
    RKR_REQUIRE(check_dim >= 0 && check_dim <= ix->dim, "check_dim %d outside [0, %d]", check_dim, ix->dim);
    RKR_TRY(ensure_device(ix));
    ix->check_dim = check_dim;
    return refine_prepare_norms(ix);
}

int rkr_index_load_sample_search(rkr_index *ix, const int32_t *sample_rank, int32_t n_sample, const float *thresholds) {
    RKR_REQUIRE(ix && sample_rank && thresholds, "null argument");
    // SampleSearch ctor: 0 < n_sample < n_data_item (SampleSearch.hpp:35-38)
    RKR_REQUIRE(n_sample > 0 && n_sample < ix->n_item, "n_sample %d must be in (0, n_item)", n_sample);
    RKR_REQUIRE(n_sample <= 0xfffe, "n_sample %d too large", n_sample);
    for (int j = 0; j < n_sample; j++) {
        RKR_REQUIRE(sample_rank[j] >= 0 && sample_rank[j] < ix->n_item, "sample rank %d out of range", sample_rank[j]);
        RKR_REQUIRE(j == 0 || sample_rank[j] >= sample_rank[j - 1], "sample ranks must be ascending");
    }
    RKR_TRY(ensure_device(ix));
    RKR_TRY(ix->sample_rank.ensure(sizeof(int32_t) * n_sample));
    RKR_TRY(ix->thr.ensure(sizeof(float) * (size_t) ix->n_user * n_sample));
    RKR_CUDA(cudaMemcpyAsync(ix->sample_rank.p, sample_rank, sizeof(int32_t) * n_sample, cudaMemcpyHostToDevice, ix->stream));
    RKR_CUDA(cudaMemcpyAsync(ix->thr.p, thresholds, sizeof(float) * (size_t) ix->n_user * n_sample, cudaMemcpyHostToDevice,
                             ix->stream));
    ix->n_sample = n_sample;
    RKR_TRY(thr_summary_build(ix));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    ix->h_sample_rank.assign(sample_rank, sample_rank + n_sample);
    return RKR_OK;
}

int rkr_index_build_sample_search(rkr_index *ix, const int32_t *sample_rank, int32_t n_sample, float *thresholds_out) {
    RKR_REQUIRE(ix && sample_rank, "null argument");
    RKR_REQUIRE(n_sample > 0 && n_sample < ix->n_item && n_sample <= 0xfffe, "n_sample %d must be in (0, n_item)",
                n_sample);
    for (int j = 0; j < n_sample; j++) {
        RKR_REQUIRE(sample_rank[j] >= 0 && sample_rank[j] < ix->n_item, "sample rank %d out of range", sample_rank[j]);
        RKR_REQUIRE(j == 0 || sample_rank[j] >= sample_rank[j - 1], "sample ranks must be ascending");
    }
    RKR_TRY(build_sample_search(ix, sample_rank, n_sample));
    if (thresholds_out) {
        RKR_CUDA(cudaMemcpy(thresholds_out, ix->thr.p, sizeof(float) * (size_t) ix->n_user * n_sample,
                            cudaMemcpyDeviceToHost));
    }
    return RKR_OK;
}

int rkr_index_load_regression(rkr_index *ix, const int32_t *sample_rank, int32_t n_sample, const float *records) {
    RKR_REQUIRE(ix && sample_rank && records, "null argument");
    RKR_REQUIRE(n_sample > 0 && n_sample <= 0xfffd, "n_sample %d out of range", n_sample);
    for (int j = 0; j < n_sample; j++) {
        RKR_REQUIRE(sample_rank[j] >= 0 && sample_rank[j] <= ix->n_item, "regression sample rank %d out of range",
                    sample_rank[j]);
        RKR_REQUIRE(j == 0 || sample_rank[j] >= sample_rank[j - 1], "regression sample ranks must be ascending");
    }
    RKR_TRY(ensure_device(ix));
    std::vector<float> rec8((size_t) ix->n_user * 8, 0.0f);
    for (int64_t u = 0; u < ix->n_user; u++) std::memcpy(&rec8[u * 8], records + u * 7, 7 * sizeof(float));
    RKR_TRY(ix->reg_rank.ensure(sizeof(int32_t) * n_sample));
    RKR_TRY(ix->reg.ensure(sizeof(float) * rec8.size()));
    RKR_CUDA(cudaMemcpyAsync(ix->reg_rank.p, sample_rank, sizeof(int32_t) * n_sample, cudaMemcpyHostToDevice, ix->stream));
    RKR_CUDA(cudaMemcpyAsync(ix->reg.p, rec8.data(), sizeof(float) * rec8.size(), cudaMemcpyHostToDevice, ix->stream));
    ix->n_sample_reg = n_sample;
    RKR_TRY(level_tables_build(ix));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

int rkr_index_load_svd(rkr_index *ix, int32_t check_dim, const float *transfer_item, const float *svd_user) {
    RKR_REQUIRE(ix && transfer_item && svd_user, "null argument");
    RKR_REQUIRE(check_dim >= 0 && check_dim <= ix->dim, "check_dim %d outside [0, %d]", check_dim, ix->dim);
    RKR_TRY(ensure_device(ix));
    const size_t d = (size_t) ix->dim;
    RKR_TRY(ix->transfer_item.ensure(sizeof(float) * d * d));
    RKR_TRY(ix->svd_user.ensure(sizeof(float) * (size_t) ix->n_user * d));
    RKR_CUDA(cudaMemcpyAsync(ix->transfer_item.p, transfer_item, sizeof(float) * d * d, cudaMemcpyHostToDevice, ix->stream));
    RKR_CUDA(cudaMemcpyAsync(ix->svd_user.p, svd_user, sizeof(float) * (size_t) ix->n_user * d, cudaMemcpyHostToDevice,
                             ix->stream));
    RKR_TRY(ix->svd_user_km.ensure(sizeof(float) * d * (size_t) kmajor_ld(ix->n_user)));
    RKR_TRY(to_kmajor(ix->svd_user.as<float>(), nullptr, ix->n_user, (int) d, ix->svd_user_km.as<float>(), ix->stream));
    ix->has_svd = true;
    ix->check_dim = check_dim;
    ix->sc_key_split = -2;  // the SVD users changed: rebuild their digit tiles on next use
    return refine_prepare_norms(ix);
}

int rkr_index_svd_read(const rkr_index *ix, float *transfer_item_out, float *svd_user_out, int32_t *check_dim_out) {
    RKR_REQUIRE(ix, "null index");
    if (!ix->has_svd) {
        set_error("the index has no SVD transform");
        return RKR_ERR_STATE;
    }
    RKR_TRY(ensure_device(ix));
    const size_t d = (size_t) ix->dim;
    if (transfer_item_out)
        RKR_CUDA(cudaMemcpy(transfer_item_out, ix->transfer_item.p, sizeof(float) * d * d, cudaMemcpyDeviceToHost));
    if (svd_user_out)
        RKR_CUDA(cudaMemcpy(svd_user_out, ix->svd_user.p, sizeof(float) * d * (size_t) ix->n_user, cudaMemcpyDeviceToHost));
    if (check_dim_out) *check_dim_out = ix->check_dim;
    return RKR_OK;
}

int rkr_index_reset_state(rkr_index *ix) {
    RKR_REQUIRE(ix, "null index");
    RKR_TRY(ensure_device(ix));
    RKR_CUDA(cudaMemsetAsync(ix->qip_state.p, 0, sizeof(float) * ix->n_user, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

int rkr_index_shape(const rkr_index *ix, int64_t *n_user, int64_t *n_item, int32_t *dim) {
    RKR_REQUIRE(ix, "null index");
    if (n_user) *n_user = ix->n_user;
    if (n_item) *n_item = ix->n_item;
    if (dim) *dim = ix->dim;
    return RKR_OK;
}

int rkr_index_size_bytes(const rkr_index *ix, uint64_t *bytes) {
    RKR_REQUIRE(ix && bytes, "null argument");
    uint64_t s = 0;
    for (const DevBuf *b : {&ix->user, &ix->item, &ix->item_sorted, &ix->item_norm, &ix->item_rnorm, &ix->user_rnorm,
                            &ix->sample_rank, &ix->thr, &ix->thr_summ, &ix->reg_rank, &ix->reg, &ix->lvt, &ix->transfer_item,
                            &ix->svd_user, &ix->svd_user_km, &ix->user_km, &ix->item_km, &ix->item_sorted_km, &ix->svd_unorm,
                            &ix->qip_state, &ix->sc_user_split, &ix->sc_umeta_split, &ix->sc_user_full,
                            &ix->sc_umeta_full, &ix->ri_item_split, &ix->ri_imeta_split, &ix->ri_item_full,
                            &ix->ri_imeta_full})
        s += b->bytes;
    *bytes = s;
    return RKR_OK;
}

static int check_query_args(rkr_index *ix, int32_t method, int32_t n_query, int32_t topk, int32_t *n_answered,
                            bool shard_call = false) {
    RKR_REQUIRE(ix, "null index");
    if (ix->sharded() != shard_call) {
        set_error(ix->sharded() ? "the index is a user shard: query it with rkr_shard_query"
                                : "rkr_shard_query: the index is not a user shard (rkr_index_set_shard)");
        return RKR_ERR_STATE;
    }
    RKR_REQUIRE(method == RKR_METHOD_QS || method == RKR_METHOD_QSRP_NORMAL_LP || method == RKR_METHOD_US,
                "unknown method %d", method);
    RKR_REQUIRE(n_query >= 0, "negative n_query");
    // QS.hpp:116-119: "top-k is too large"; topk < 1 leaves the reference's heaps empty.
    RKR_REQUIRE(topk >= 1 && topk <= ix->n_user_all(), "topk %d outside [1, n_user=%lld]", topk,
                (long long) ix->n_user_all());
    RKR_REQUIRE(topk <= 4096, "topk %d above the supported maximum of 4096", topk);
    if (ix->n_sample <= 0) {
        set_error("method needs the sampled-threshold index (load or build it first)");
        return RKR_ERR_STATE;
    }
    if (method != RKR_METHOD_US && ix->check_dim < 0) {
        set_error("method needs check_dim (rkr_index_set_check_dim or rkr_index_load_svd)");
        return RKR_ERR_STATE;
    }
    if (method == RKR_METHOD_QSRP_NORMAL_LP && (!ix->has_svd || ix->n_sample_reg <= 0)) {
        set_error("QSRPNormalLP needs the SVD transform and the regression models");
        return RKR_ERR_STATE;
    }
    int nq = n_query;
    if (method == RKR_METHOD_US && ix->n_sample <= 1000) {  // US.hpp:113
        RKR_REQUIRE(n_query >= 100, "US with n_sample <= 1000 answers exactly 100 queries; got %d", n_query);
        nq = 100;
    }
    if (n_answered) *n_answered = nq;
    return RKR_OK;
}

int rkr_retrieval_device(rkr_index *ix, int32_t method, const float *d_query, int32_t n_query, int32_t topk,
                         rkr_user_rank *d_out, rkr_query_stats *d_stats, int32_t *n_answered, void *stream) {
    int32_t nq = 0;
    RKR_TRY(check_query_args(ix, method, n_query, topk, &nq));
    if (n_answered) *n_answered = nq;
    if (nq == 0) return RKR_OK;
    RKR_REQUIRE(d_query && d_out, "null query/output pointer");
    RKR_TRY(ensure_device(ix));
    cudaStream_t st = stream ? (cudaStream_t) stream : ix->stream;
    BatchSpec bs;
    bs.topk = topk;
    return query_batch(ix, method, d_query, nq, bs, d_out, d_stats, st);
}

int rkr_retrieval(rkr_index *ix, int32_t method, const float *query, int32_t n_query, int32_t topk, rkr_user_rank *out,
                  rkr_query_stats *stats, int32_t *n_answered) {
    int32_t nq = 0;
    RKR_TRY(check_query_args(ix, method, n_query, topk, &nq));
    if (n_answered) *n_answered = nq;
    if (nq == 0) return RKR_OK;
    RKR_REQUIRE(query && out, "null query/output pointer");
    RKR_TRY(ensure_device(ix));
    const size_t qb = sizeof(float) * (size_t) nq * ix->dim;
    const size_t ob = sizeof(rkr_user_rank) * (size_t) nq * topk;
    const size_t sb = sizeof(rkr_query_stats) * (size_t) nq;
    RKR_TRY(ix->ws_query.ensure(qb));
    RKR_TRY(ix->ws_out.ensure(ob));
    RKR_TRY(ix->ws_stats.ensure(sb));
    RKR_CUDA(cudaMemcpyAsync(ix->ws_query.p, query, qb, cudaMemcpyHostToDevice, ix->stream));
    BatchSpec bs;
    bs.topk = topk;
    RKR_TRY(query_batch(ix, method, ix->ws_query.as<float>(), nq, bs, ix->ws_out.as<rkr_user_rank>(),
                        stats ? ix->ws_stats.as<rkr_query_stats>() : nullptr, ix->stream));
    RKR_CUDA(cudaMemcpyAsync(out, ix->ws_out.p, ob, cudaMemcpyDeviceToHost, ix->stream));
    if (stats) RKR_CUDA(cudaMemcpyAsync(stats, ix->ws_stats.p, sb, cudaMemcpyDeviceToHost, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

// Per-query top-k: every k in [1, min(n_user, 4096)]; returns the total output entries of the
// answered queries in *n_out.
static int check_k_per_q(rkr_index *ix, const int32_t *k_per_q, int32_t n, int64_t *n_out) {
    RKR_REQUIRE(k_per_q || n == 0, "null k_per_q");
    int64_t s = 0;
    for (int32_t q = 0; q < n; q++) {
        const int32_t k = k_per_q[q];
        RKR_REQUIRE(k >= 1 && k <= ix->n_user_all(), "k_per_q[%d] = %d outside [1, n_user=%lld]", q, k,
                    (long long) ix->n_user_all());
        RKR_REQUIRE(k <= 4096, "k_per_q[%d] = %d above the supported maximum of 4096", q, k);
        s += k;
    }
    *n_out = s;
    return RKR_OK;
}

int rkr_query_device(rkr_index *ix, int32_t method, const float *d_query, int32_t n_query, const int32_t *k_per_q,
                     rkr_user_rank *d_out, rkr_query_stats *d_stats, int32_t *n_answered, void *stream) {
    int32_t nq = 0;
    RKR_TRY(check_query_args(ix, method, n_query, 1, &nq));
    if (n_answered) *n_answered = nq;
    if (nq == 0) return RKR_OK;
    int64_t n_out = 0;
    RKR_TRY(check_k_per_q(ix, k_per_q, nq, &n_out));
    RKR_REQUIRE(d_query && d_out, "null query/output pointer");
    RKR_TRY(ensure_device(ix));
    cudaStream_t st = stream ? (cudaStream_t) stream : ix->stream;
    BatchSpec bs;
    bs.k = k_per_q;
    return query_batch(ix, method, d_query, nq, bs, d_out, d_stats, st);
}

int rkr_query(rkr_index *ix, int32_t method, const float *query, int32_t n_query, const int32_t *k_per_q,
              rkr_user_rank *out, rkr_query_stats *stats, int32_t *n_answered) {
    int32_t nq = 0;
    RKR_TRY(check_query_args(ix, method, n_query, 1, &nq));
    if (n_answered) *n_answered = nq;
    if (nq == 0) return RKR_OK;
    int64_t n_out = 0;
    RKR_TRY(check_k_per_q(ix, k_per_q, nq, &n_out));
    RKR_REQUIRE(query && out, "null query/output pointer");
    RKR_TRY(ensure_device(ix));
    const size_t qb = sizeof(float) * (size_t) nq * ix->dim;
    const size_t ob = sizeof(rkr_user_rank) * (size_t) n_out;
    const size_t sb = sizeof(rkr_query_stats) * (size_t) nq;
    RKR_TRY(ix->ws_query.ensure(qb));
    RKR_TRY(ix->ws_out.ensure(ob));
    RKR_TRY(ix->ws_stats.ensure(sb));
    RKR_CUDA(cudaMemcpyAsync(ix->ws_query.p, query, qb, cudaMemcpyHostToDevice, ix->stream));
    BatchSpec bs;
    bs.k = k_per_q;
    RKR_TRY(query_batch(ix, method, ix->ws_query.as<float>(), nq, bs, ix->ws_out.as<rkr_user_rank>(),
                        stats ? ix->ws_stats.as<rkr_query_stats>() : nullptr, ix->stream));
    RKR_CUDA(cudaMemcpyAsync(out, ix->ws_out.p, ob, cudaMemcpyDeviceToHost, ix->stream));
    if (stats) RKR_CUDA(cudaMemcpyAsync(stats, ix->ws_stats.p, sb, cudaMemcpyDeviceToHost, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

int rkr_index_set_shard(rkr_index *ix, int32_t shard, int32_t n_shards, int64_t user_offset, int64_t n_user_total,
                        rkr_exchange_fn exchange, void *ctx) {
    RKR_REQUIRE(ix, "null index");
    RKR_REQUIRE(n_shards >= 1 && shard >= 0 && shard < n_shards, "shard %d of %d", shard, n_shards);
    if (n_shards == 1 && !exchange) {  // whole again
        RKR_REQUIRE(user_offset == 0 && (n_user_total == 0 || n_user_total == ix->n_user),
                    "a whole index starts at user 0 and holds n_user_total users");
        ix->shard = rkr_index::Shard();
        return RKR_OK;
    }
    RKR_REQUIRE(exchange, "a user shard needs an exchange function");
    RKR_REQUIRE(user_offset >= 0 && user_offset + ix->n_user <= n_user_total,
                "users [%lld, %lld) outside [0, n_user_total=%lld)", (long long) user_offset,
                (long long) (user_offset + ix->n_user), (long long) n_user_total);
    RKR_REQUIRE(n_user_total <= INT32_MAX, "n_user_total %lld above the 32-bit user ids", (long long) n_user_total);
    ix->shard.index = shard;
    ix->shard.count = n_shards;
    ix->shard.user_offset = user_offset;
    ix->shard.n_user_total = n_user_total;
    ix->shard.fn = exchange;
    ix->shard.ctx = ctx;
    return RKR_OK;
}

int rkr_shard_query(rkr_index *ix, int32_t method, const float *query, int32_t n_query, const int32_t *k_per_q,
                    rkr_user_rank *part, int32_t *n_front, rkr_query_stats *stats, int32_t *n_answered) {
    int32_t nq = 0;
    RKR_TRY(check_query_args(ix, method, n_query, 1, &nq, true));
    if (n_answered) *n_answered = nq;
    if (nq == 0) return RKR_OK;
    int64_t n_out = 0;
    RKR_TRY(check_k_per_q(ix, k_per_q, nq, &n_out));
    RKR_REQUIRE(query && part && n_front, "null query/part/n_front pointer");
    RKR_TRY(ensure_device(ix));
    const size_t qb = sizeof(float) * (size_t) nq * ix->dim;
    const size_t ob = sizeof(rkr_user_rank) * (size_t) n_out;
    const size_t sb = sizeof(rkr_query_stats) * (size_t) nq;
    RKR_TRY(ix->ws_query.ensure(qb));
    RKR_TRY(ix->ws_out.ensure(ob));
    RKR_TRY(ix->ws_stats.ensure(sb));
    RKR_CUDA(cudaMemcpyAsync(ix->ws_query.p, query, qb, cudaMemcpyHostToDevice, ix->stream));
    BatchSpec bs;
    bs.k = k_per_q;
    bs.front = n_front;
    RKR_TRY(query_batch(ix, method, ix->ws_query.as<float>(), nq, bs, ix->ws_out.as<rkr_user_rank>(),
                        stats ? ix->ws_stats.as<rkr_query_stats>() : nullptr, ix->stream));
    RKR_CUDA(cudaMemcpyAsync(part, ix->ws_out.p, ob, cudaMemcpyDeviceToHost, ix->stream));
    if (stats) RKR_CUDA(cudaMemcpyAsync(stats, ix->ws_stats.p, sb, cudaMemcpyDeviceToHost, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

int rkr_score_estimates(rkr_index *ix, int32_t method, const float *query, int32_t n_query, float *out) {
    int32_t nq = 0;
    RKR_TRY(check_query_args(ix, method, n_query, 1, &nq));
    RKR_REQUIRE(method != RKR_METHOD_US, "rkr_score_estimates: QS or QSRPNormalLP");
    RKR_REQUIRE(nq >= 1 && nq <= kMaxChunkQueries && query && out, "rkr_score_estimates: 1 .. %d queries",
                kMaxChunkQueries);
    RKR_TRY(ensure_device(ix));
    const size_t qb = sizeof(float) * (size_t) nq * ix->dim;
    const size_t db = sizeof(float2) * (size_t) nq * (size_t) ix->n_user;
    DevBuf dump;
    RKR_TRY(dump.ensure(db));
    RKR_TRY(ix->ws_query.ensure(qb));
    RKR_TRY(ix->ws_out.ensure(sizeof(rkr_user_rank) * (size_t) nq));
    RKR_CUDA(cudaMemcpyAsync(ix->ws_query.p, query, qb, cudaMemcpyHostToDevice, ix->stream));
    RKR_CUDA(cudaMemsetAsync(dump.p, 0xff, db, ix->stream));  // NaN where the tensor cores did not run
    // one pass of the pipeline with the scores kernel writing its estimates; the state it carries is
    // put back afterwards
    std::vector<float> state((size_t) ix->n_user);
    RKR_CUDA(cudaMemcpyAsync(state.data(), ix->qip_state.p, sizeof(float) * state.size(), cudaMemcpyDeviceToHost,
                             ix->stream));
    ix->score_dump = dump.as<float2>();
    const bool graphs = ix->graphs_on;
    ix->graphs_on = false;
    BatchSpec bs;
    bs.topk = 1;
    const int rc = query_batch(ix, method, ix->ws_query.as<float>(), nq, bs, ix->ws_out.as<rkr_user_rank>(), nullptr,
                               ix->stream);
    ix->score_dump = nullptr;
    ix->graphs_on = graphs;
    RKR_TRY(rc);
    RKR_CUDA(cudaMemcpyAsync(ix->qip_state.p, state.data(), sizeof(float) * state.size(), cudaMemcpyHostToDevice,
                             ix->stream));
    RKR_CUDA(cudaMemcpyAsync(out, dump.p, db, cudaMemcpyDeviceToHost, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    dump.release();
    return RKR_OK;
}

int rkr_score_sort_batch(rkr_index *ix, int64_t start_user, int64_t n_rows, float *rows_out) {
    RKR_REQUIRE(ix && rows_out, "null argument");
    RKR_REQUIRE(start_user >= 0 && n_rows >= 0 && start_user + n_rows <= ix->n_user, "user range out of bounds");
    if (n_rows == 0) return RKR_OK;
    return score_sort_rows(ix, start_user, n_rows, rows_out);
}

int rkr_index_query_rank_distribution(rkr_index *ix, const int32_t *sample_item, int32_t n_sample_item,
                                      int32_t *accu_out) {
    RKR_REQUIRE(ix && sample_item && accu_out, "null argument");
    RKR_REQUIRE(n_sample_item > 0 && n_sample_item <= ix->n_item, "n_sample_item %d out of range", n_sample_item);
    for (int s = 0; s < n_sample_item; s++)
        RKR_REQUIRE(sample_item[s] >= 0 && sample_item[s] < ix->n_item, "sample item %d out of range", sample_item[s]);
    return query_rank_distribution(ix, sample_item, n_sample_item, accu_out);
}

int rkr_profile_enable(rkr_index *ix, int32_t on) {
    RKR_REQUIRE(ix, "null index");
    RKR_TRY(ensure_device(ix));
    ix->prof.resolve();
    ix->prof.on = on != 0;
    return RKR_OK;
}

int rkr_profile_read(rkr_index *ix, int32_t max_kernels, char *names, double *total_ms, int64_t *launches,
                     int32_t *n_kernels) {
    RKR_REQUIRE(ix && n_kernels, "null argument");
    RKR_TRY(ensure_device(ix));
    ix->prof.resolve();
    const int n = (int) ix->prof.names.size();
    *n_kernels = n;
    for (int i = 0; i < n && i < max_kernels; i++) {
        if (names) {
            std::strncpy(names + (size_t) i * 64, ix->prof.names[i].c_str(), 63);
            names[(size_t) i * 64 + 63] = 0;
        }
        if (total_ms) total_ms[i] = ix->prof.total_ms[i];
        if (launches) launches[i] = ix->prof.launches[i];
    }
    if (max_kernels >= n)  // a size query (max_kernels < n) leaves the counters in place
        for (int i = 0; i < n; i++) { ix->prof.total_ms[i] = 0; ix->prof.launches[i] = 0; }
    return RKR_OK;
}

}  // extern "C"
