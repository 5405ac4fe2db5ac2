// The SVD transform built on the device from the index's resident users (SVD::PerformSVD,
// SVD.hpp:62-124): the Gram matrix user^T user in double on the device, its eigen-decomposition on
// the host (svd_from_gram, rkr_host.cpp: d x d, d <= a few hundred), and the projection
// svd_user = user Es diag(1/s) on the device with the host projection's operations (each output
// summed over the coordinates in order, one rounding per operation).  As rkr_svd_build, a valid
// transform, not the reference's bits (the reference's SVD comes from LAPACK); query parity is
// defined on a given SVD index.
#include <vector>

#include "rkr_internal.cuh"
#include "rkr_svd_host.h"

namespace rkr {
namespace {

constexpr int kGramUsers = 4096;  // users per block of the Gram pass

// One 32 x 32 tile (rows p0.., columns q0.., p0 <= q0) of the Gram matrix over one chunk of users:
// 32 users' two column slices staged in shared memory as doubles, four outputs per thread; the
// chunk's sums go to its own slice of `part` ([chunk][d][d]), summed in chunk order afterwards, so
// the matrix is the same on every run.
__global__ void __launch_bounds__(256) gram_kernel(const float *__restrict__ user, int64_t n_user, int d,
                                                   const int2 *__restrict__ tiles, double *__restrict__ part) {
    __shared__ double sp[32][33], sq[32][33];
    const int2 tl = tiles[blockIdx.x];
    const int p0 = tl.x * 32, q0 = tl.y * 32;
    const int64_t u0 = (int64_t) blockIdx.y * kGramUsers;
    const int64_t u1 = min(n_user, u0 + kGramUsers);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t ub = u0; ub < u1; ub += 32) {
        for (int r = ty; r < 32; r += 8) {
            const int64_t u = ub + r;
            sp[r][tx] = (u < u1 && p0 + tx < d) ? (double) __ldg(user + u * d + p0 + tx) : 0.0;
            sq[r][tx] = (u < u1 && q0 + tx < d) ? (double) __ldg(user + u * d + q0 + tx) : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int r = 0; r < 32; r++) {
            const double b = sq[r][tx];
#pragma unroll
            for (int m = 0; m < 4; m++) acc[m] = fma(sp[r][ty + 8 * m], b, acc[m]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int p = p0 + ty + 8 * m, q = q0 + tx;
        if (p < d && q < d && p <= q) part[(size_t) blockIdx.y * d * d + (size_t) p * d + q] = acc[m];
    }
}

// G[e] = the chunks' partial sums of entry e added in chunk order (upper triangle).
__global__ void gram_sum_kernel(const double *__restrict__ part, int n_chunks, int d, double *__restrict__ G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d * d) return;
    const int p = e / d, q = e % d;
    if (p > q) return;
    double s = 0.0;
    for (int c = 0; c < n_chunks; c++) s += part[(size_t) c * d * d + e];
    G[e] = s;
}

// svd_user[u][k] = user[u] . Es[:, k] / s[k] (0 where s[k] is 0), summed over the coordinates in
// order as the host projection sums them.
__global__ void __launch_bounds__(256) project_kernel(const float *__restrict__ user, int64_t n_user, int d,
                                                      const double *__restrict__ Es, const float *__restrict__ s,
                                                      float *__restrict__ svd_user) {
    const int64_t total = n_user * d;
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int64_t u = idx / d;
        const int k = (int) (idx - u * d);
        const float *ur = user + u * d;
        double acc = 0.0;
        for (int i = 0; i < d; i++) acc = __dadd_rn(acc, __dmul_rn((double) __ldg(ur + i), __ldg(Es + (size_t) i * d + k)));
        const float sk = s[k];
        svd_user[idx] = sk > 0 ? __double2float_rn(__ddiv_rn(acc, (double) sk)) : 0.0f;
    }
}

}  // namespace
}  // namespace rkr

namespace rkr {

int svd_build_device(rkr_index *ix, float sigma_ratio, float *transfer_item_out, float *svd_user_out,
                     int32_t *check_dim_out) {
    const int d = ix->dim;
    const int64_t U = ix->n_user;
    cudaStream_t st = ix->stream;
    // Gram matrix: the upper-triangle tiles over user chunks
    const int nt = (d + 31) / 32;
    std::vector<int2> tiles;
    for (int a = 0; a < nt; a++)
        for (int b = a; b < nt; b++) tiles.push_back(make_int2(a, b));
    struct Scratch {  // released on every return
        DevBuf b[4];
        ~Scratch() { for (auto &x : b) x.release(); }
    } scratch;
    DevBuf &g = scratch.b[0], &tl = scratch.b[1], &es = scratch.b[2], &sv = scratch.b[3];
    const int n_chunks = (int) ((U + kGramUsers - 1) / kGramUsers);
    RKR_TRY(g.ensure(sizeof(double) * (size_t) d * d * (size_t) (n_chunks + 1)));
    double *part = g.as<double>() + (size_t) d * d;  // [n_chunks][d][d]; the sums at the front
    RKR_TRY(tl.ensure(sizeof(int2) * tiles.size()));
    RKR_CUDA(cudaMemsetAsync(g.p, 0, sizeof(double) * (size_t) d * d, st));
    RKR_CUDA(cudaMemcpyAsync(tl.p, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, st));
    const dim3 gg((unsigned) tiles.size(), (unsigned) n_chunks);
    timed(ix, st, "svd_gram", [&] { gram_kernel<<<gg, 256, 0, st>>>(ix->user.as<float>(), U, d, tl.as<int2>(), part); });
    RKR_CUDA(cudaGetLastError());
    gram_sum_kernel<<<(unsigned) ((d * d + 255) / 256), 256, 0, st>>>(part, n_chunks, d, g.as<double>());
    RKR_CUDA(cudaGetLastError());
    std::vector<double> G((size_t) d * d);
    RKR_CUDA(cudaMemcpyAsync(G.data(), g.p, sizeof(double) * G.size(), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < d; i++)
        for (int j = 0; j < i; j++) G[(size_t) i * d + j] = G[(size_t) j * d + i];
    std::vector<float> ti((size_t) d * d), s;
    std::vector<double> Es;
    int check_dim = 0;
    svd_from_gram(G, d, sigma_ratio, ti.data(), Es, s, &check_dim);
    // projection into the index's SVD-space users
    RKR_TRY(es.ensure(sizeof(double) * Es.size()));
    RKR_TRY(sv.ensure(sizeof(float) * s.size()));
    RKR_CUDA(cudaMemcpyAsync(es.p, Es.data(), sizeof(double) * Es.size(), cudaMemcpyHostToDevice, st));
    RKR_CUDA(cudaMemcpyAsync(sv.p, s.data(), sizeof(float) * s.size(), cudaMemcpyHostToDevice, st));
    RKR_TRY(ix->svd_user.ensure(sizeof(float) * (size_t) U * d));
    RKR_TRY(ix->transfer_item.ensure(sizeof(float) * (size_t) d * d));
    RKR_CUDA(cudaMemcpyAsync(ix->transfer_item.p, ti.data(), sizeof(float) * ti.size(), cudaMemcpyHostToDevice, st));
    timed(ix, st, "svd_project", [&] {
        project_kernel<<<148 * 16, 256, 0, st>>>(ix->user.as<float>(), U, d, es.as<double>(), sv.as<float>(),
                                                 ix->svd_user.as<float>());
    });
    RKR_CUDA(cudaGetLastError());
    // the rest of rkr_index_load_svd: the k-major copy, check_dim, digit tiles rebuilt on next use
    RKR_TRY(ix->svd_user_km.ensure(sizeof(float) * (size_t) d * (size_t) kmajor_ld(U)));
    RKR_TRY(to_kmajor(ix->svd_user.as<float>(), nullptr, U, d, ix->svd_user_km.as<float>(), st));
    ix->has_svd = true;
    ix->check_dim = check_dim;
    ix->sc_key_split = -2;
    RKR_TRY(refine_prepare_norms(ix));
    if (transfer_item_out) std::copy(ti.begin(), ti.end(), transfer_item_out);
    if (svd_user_out)
        RKR_CUDA(cudaMemcpyAsync(svd_user_out, ix->svd_user.p, sizeof(float) * (size_t) U * d, cudaMemcpyDeviceToHost, st));
    if (check_dim_out) *check_dim_out = check_dim;
    RKR_CUDA(cudaStreamSynchronize(st));
    return RKR_OK;
}

}  // namespace rkr

extern "C" int rkr_index_svd_build(rkr_index *ix, float sigma_ratio, float *transfer_item_out, float *svd_user_out,
                                   int32_t *check_dim_out) {
    RKR_REQUIRE(ix, "null index");
    RKR_REQUIRE(sigma_ratio > 0.0f && sigma_ratio <= 1.0f, "sigma_ratio %g outside (0, 1]", (double) sigma_ratio);
    if (ix->sharded()) {
        // every shard needs the same transform, built over every user
        ::rkr::set_error("rkr_index_svd_build: the index is a user shard (build the transform over all users, "
                         "rkr_svd_build, and load each shard's rows)");
        return RKR_ERR_STATE;
    }
    RKR_TRY(rkr::ensure_device(ix));
    return rkr::svd_build_device(ix, sigma_ratio, transfer_item_out, svd_user_out, check_dim_out);
}
