// User insertion and deletion against a built index: QSRPNormalLPUpdate::InsertUser / DeleteUser
// (src/impl/Update/QSRPNormalLPUpdate.hpp:308-365).  An insertion appends the users with their
// sampled thresholds (SampleSearchUpdate::InsertUser, SampleSearchUpdate.hpp:72-87: the new users'
// sorted score rows sampled at the index's ranks) and regression models
// (NormalLinearRegressionLPUpdate::InsertUser), all computed on the device, and rebuilds the SVD
// transform over every user (SVDUpdate::InsertUser, SVDUpdate.hpp:63-79, then PartDimPartNorm's norms
// for the new check_dim).  A deletion drops the users' rows from every per-user array and keeps the
// transform (SVDUpdate::DeleteUser, :81-84).  Both resize the carried QSRPNormalLP scores as the
// reference resizes queryIP_l_ (a std::vector resize: new users start at zero; a deletion keeps the
// first n_user entries, whoever they belonged to).  Item updates (the rank-offset searches of
// SampleSearchUpdate::SearchInsertDelete) are not built.
#include <algorithm>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {
namespace {

// b holds `keep` bytes that must survive; after this it holds at least `want` bytes.
int grow_keep(DevBuf &b, size_t keep, size_t want, cudaStream_t st) {
    if (want <= b.bytes) return RKR_OK;
    DevBuf n;
    RKR_TRY(n.ensure(want));
    if (keep) RKR_CUDA(cudaMemcpyAsync(n.p, b.p, keep, cudaMemcpyDeviceToDevice, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    b.release();
    b = n;
    return RKR_OK;
}

// dst row i = src row keep[i], w floats per row.
__global__ void keep_rows_kernel(const float *__restrict__ src, int64_t w, const int64_t *__restrict__ keep,
                                 int64_t n_keep, float *__restrict__ dst) {
    const int64_t total = n_keep * w;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t) gridDim.x * blockDim.x) {
        const int64_t r = i / w, c = i - r * w;
        dst[i] = src[keep[r] * w + c];
    }
}

// The rows `keep` of b ([n][w] floats) in a new buffer of their own.
int keep_rows(DevBuf &b, int64_t w, const int64_t *d_keep, int64_t n_keep, cudaStream_t st) {
    if (!b.p) return RKR_OK;
    DevBuf n;
    RKR_TRY(n.ensure(sizeof(float) * (size_t) (n_keep * w)));
    const int64_t total = n_keep * w;
    keep_rows_kernel<<<(unsigned) std::min<int64_t>(148 * 16, (total + 255) / 256), 256, 0, st>>>(
        b.as<float>(), w, d_keep, n_keep, n.as<float>());
    RKR_CUDA(cudaGetLastError());
    RKR_CUDA(cudaStreamSynchronize(st));
    b.release();
    b = n;
    return RKR_OK;
}

// What depends on every user's rows: the k-major copies, the threshold summaries, the level tables,
// the refinement norms; the cached digit tiles of the users and the captured phase-1 graphs go.
int users_changed(rkr_index *ix) {
    const int d = ix->dim;
    const int64_t U = ix->n_user;
    cudaStream_t st = ix->stream;
    RKR_TRY(ix->user_km.ensure(sizeof(float) * (size_t) d * (size_t) kmajor_ld(U)));
    RKR_TRY(to_kmajor(ix->user.as<float>(), nullptr, U, d, ix->user_km.as<float>(), st));
    if (ix->has_svd) {
        RKR_TRY(ix->svd_user_km.ensure(sizeof(float) * (size_t) d * (size_t) kmajor_ld(U)));
        RKR_TRY(to_kmajor(ix->svd_user.as<float>(), nullptr, U, d, ix->svd_user_km.as<float>(), st));
    }
    if (ix->n_sample > 0) RKR_TRY(thr_summary_build(ix));
    if (ix->n_sample_reg > 0) RKR_TRY(level_tables_build(ix));
    if (ix->check_dim >= 0) RKR_TRY(refine_prepare_norms(ix));
    ix->sc_key_split = -2;
    ix->sc_key_full = -2;
    for (auto &g : ix->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    ix->graphs.clear();
    RKR_CUDA(cudaStreamSynchronize(st));
    return RKR_OK;
}

}  // namespace
}  // namespace rkr

using namespace rkr;

extern "C" {

int rkr_index_insert_users(rkr_index *ix, const float *user, int64_t n, float sigma) {
    RKR_REQUIRE(ix && user, "null argument");
    RKR_REQUIRE(n > 0 && ix->n_user + n < (int64_t(1) << 31), "n %lld out of range", (long long) n);
    RKR_REQUIRE(!ix->sharded(), "rkr_index_insert_users: the index is a user shard");
    if (ix->n_sample <= 0) {
        set_error("rkr_index_insert_users: the index has no sampled thresholds");
        return RKR_ERR_STATE;
    }
    RKR_REQUIRE(!ix->has_svd || (sigma > 0.0f && sigma <= 1.0f), "sigma %g outside (0, 1]", (double) sigma);
    RKR_TRY(ensure_device(ix));
    cudaStream_t st = ix->stream;
    const int d = ix->dim, S = ix->n_sample;
    if (ix->n_sample_reg > 0) {
        // the models are fitted from the thresholds, so they must share the sample ranks
        std::vector<int32_t> rr((size_t) ix->n_sample_reg);
        RKR_CUDA(cudaMemcpy(rr.data(), ix->reg_rank.p, sizeof(int32_t) * rr.size(), cudaMemcpyDeviceToHost));
        if (rr != ix->h_sample_rank) {
            set_error("rkr_index_insert_users: the regression models' sample ranks differ from the thresholds'");
            return RKR_ERR_STATE;
        }
    }
    const int64_t U0 = ix->n_user, U1 = U0 + n;
    RKR_TRY(grow_keep(ix->user, sizeof(float) * (size_t) (U0 * d), sizeof(float) * (size_t) (U1 * d), st));
    RKR_CUDA(cudaMemcpyAsync(ix->user.as<float>() + U0 * d, user, sizeof(float) * (size_t) (n * d), cudaMemcpyHostToDevice,
                             st));
    RKR_TRY(grow_keep(ix->qip_state, sizeof(float) * (size_t) U0, sizeof(float) * (size_t) U1, st));
    RKR_CUDA(cudaMemsetAsync(ix->qip_state.as<float>() + U0, 0, sizeof(float) * (size_t) n, st));
    RKR_TRY(grow_keep(ix->thr, sizeof(float) * (size_t) (U0 * S), sizeof(float) * (size_t) (U1 * S), st));
    ix->n_user = U1;
    // the new users' thresholds: their score rows against every item, sampled at the index's ranks
    RKR_TRY(build_thresholds_range(ix, U0, U1));
    if (ix->n_sample_reg > 0) {
        RKR_TRY(grow_keep(ix->reg, sizeof(float) * 8 * (size_t) U0, sizeof(float) * 8 * (size_t) U1, st));
        RKR_TRY(fit_regression_device(ix, U0, U1, st));
    }
    if (ix->has_svd) {
        RKR_TRY(svd_build_device(ix, sigma, nullptr, nullptr, nullptr));  // every user's rows, new check_dim
    }
    return users_changed(ix);
}

int rkr_index_delete_users(rkr_index *ix, const int64_t *ids, int64_t n) {
    RKR_REQUIRE(ix && (ids || n == 0), "null argument");
    RKR_REQUIRE(n >= 0 && n < ix->n_user, "n %lld outside [0, n_user)", (long long) n);
    RKR_REQUIRE(!ix->sharded(), "rkr_index_delete_users: the index is a user shard");
    if (n == 0) return RKR_OK;
    std::vector<int64_t> del(ids, ids + n);
    std::sort(del.begin(), del.end());
    for (int64_t i = 0; i < n; i++) {
        RKR_REQUIRE(del[i] >= 0 && del[i] < ix->n_user, "user %lld out of range", (long long) del[i]);
        RKR_REQUIRE(i == 0 || del[i] != del[i - 1], "user %lld listed twice", (long long) del[i]);
    }
    RKR_TRY(ensure_device(ix));
    cudaStream_t st = ix->stream;
    const int64_t U0 = ix->n_user, U1 = U0 - n;
    std::vector<int64_t> keep;
    keep.reserve((size_t) U1);
    for (int64_t u = 0, j = 0; u < U0; u++) {
        if (j < n && del[j] == u) { j++; continue; }
        keep.push_back(u);
    }
    DevBuf dk;
    RKR_TRY(dk.ensure(sizeof(int64_t) * keep.size()));
    RKR_CUDA(cudaMemcpyAsync(dk.p, keep.data(), sizeof(int64_t) * keep.size(), cudaMemcpyHostToDevice, st));
    int rc = keep_rows(ix->user, ix->dim, dk.as<int64_t>(), U1, st);
    if (rc == RKR_OK && ix->n_sample > 0) rc = keep_rows(ix->thr, ix->n_sample, dk.as<int64_t>(), U1, st);
    if (rc == RKR_OK && ix->n_sample_reg > 0) rc = keep_rows(ix->reg, 8, dk.as<int64_t>(), U1, st);
    if (rc == RKR_OK && ix->has_svd) rc = keep_rows(ix->svd_user, ix->dim, dk.as<int64_t>(), U1, st);
    dk.release();
    RKR_TRY(rc);
    // the carried scores: the first U1 entries stay, as a std::vector resize leaves them
    ix->n_user = U1;
    return users_changed(ix);
}

}  // extern "C"
