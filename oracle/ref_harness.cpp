// ref_harness.cpp -- drives the reference's own, unmodified hot-path headers
// (DBGroup-SUSTech/reverse-k-ranks, src/include and src/impl) through a C ABI, so the oracle
// restatement (rkr_oracle.c) and the product can be checked against the reference itself.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/librkr_ref.so from the
// reference sources where they lie; never part of the product.  Only tests/ and bench.py's
// reference / cpu_baseline legs load it.
//
// The reference needs Boost, spdlog, Eigen, sdlp and Armadillo, which this machine lacks;
// oracle/ref_shim/ stands in for the few symbols the hot path touches (logging no-ops,
// std::sort for boost's sort, an exact minimax-line solver for the one LP the regression model
// solves, a Jacobi thin SVD).  Everything else -- bound search, pruning, refinement, result
// assembly, the regression model's evaluation and its index file formats -- is the reference's
// code, compiled with strict IEEE float arithmetic (no FMA contraction), as its Debug build.
// Include order follows the query app (src/app/ReverseRankIndex.cpp:5-17): the query-path and
// regression headers are parsed before any build-side header.  This matters: the build-side
// headers include <parallel/algorithm>, which exports std::exp(float) into the global namespace,
// while the query app (and the regression app, BuildRegressionIndex.cpp) never include it, so
// there NormalLinearRegressionLP::CDFPhi's unqualified exp() is the double ::exp.
#include "util/VectorIO.hpp"
#include "util/TimeMemory.hpp"
#include "util/FileIO.hpp"
#include "struct/UserRankElement.hpp"
#include "struct/VectorMatrix.hpp"
#include "QS.hpp"
#include "QSRPNormalLP.hpp"
#include "US.hpp"
#include "util/NameTranslation.hpp"
#include "alg/RankBoundRefinement/SampleSearch.hpp"
#include "alg/RankBoundRefinement/PruneCandidateByBound.hpp"
#include "alg/RegressionPruning/NormalLinearRegressionLP.hpp"
#include "alg/SVD.hpp"
// build side (bsibc, qdibc, fsr)
#include "score_computation/ComputeScoreTableBatch.hpp"
#include "alg/RankBoundRefinement/FindSampleRank/OptimalSampleRank.hpp"
#include "alg/RankBoundRefinement/FindSampleRank/OptimalSampleRankFast.hpp"
#include "alg/RankBoundRefinement/FindSampleRank/UniformSample.hpp"
#include "QueryRankByComputation.hpp"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

using namespace ReverseMIPS;

namespace {

void fill_vm(VectorMatrix &vm, const float *src, int64_t n, int32_t d) {
    std::unique_ptr<float[]> p = std::make_unique<float[]>((size_t) n * (size_t) d);
    std::memcpy(p.get(), src, sizeof(float) * (size_t) n * (size_t) d);
    vm.init(p, (int) n, (int) d);
}

void ensure_index_dirs(const std::string &dir) {
    for (const char *sub : {"memory_index", "qrs_to_sample_index", "query_distribution", "svd_index"})
        std::filesystem::create_directories(dir + "/" + sub);
}

// Writes a SampleSearch index file in the reference's layout through the reference's own writer.
void write_sample_index(const std::string &dir, const char *ds, const char *name, const int32_t *rank,
                        int32_t S, const float *thr, int64_t n_user, int64_t n_item, int32_t nsq,
                        int32_t stopk, bool is_query_distribution) {
    std::vector<int> rank_l(rank, rank + S);
    SampleSearch ss((int) n_item, (int) n_user, rank_l, S);
    // LoopPreprocess gathers row[rank[j]]; feed it a row holding the thresholds at those positions.
    std::vector<float> row((size_t) n_item);
    for (int64_t u = 0; u < n_user; u++) {
        for (int j = 0; j < S; j++) row[rank[j]] = thr[u * S + j];
        ss.LoopPreprocess(row.data(), (int) u);
    }
    ss.SaveIndex(dir.c_str(), ds, name, true, is_query_distribution, nsq, stopk);
}

void write_svd_index(const std::string &dir, const char *ds, int64_t n_user, int64_t n_item, int32_t d,
                     int32_t check_dim, const float *transfer_item, const float *svd_user) {
    char path[512];
    std::snprintf(path, sizeof path, "%s/svd_index/%s.index", dir.c_str(), ds);
    std::ofstream o(path, std::ios::binary);
    size_t nu = (size_t) n_user, ni = (size_t) n_item, vd = (size_t) d;
    float sigma = 0.7f;
    int cd = check_dim;
    o.write((char *) &nu, sizeof nu); o.write((char *) &ni, sizeof ni); o.write((char *) &vd, sizeof vd);
    o.write((char *) &sigma, sizeof sigma); o.write((char *) &cd, sizeof cd);
    o.write((const char *) transfer_item, (std::streamsize) (sizeof(float) * vd * vd));
    o.write((const char *) svd_user, (std::streamsize) (sizeof(float) * nu * vd));
    std::vector<float> zero(ni * vd, 0.0f);  // transfer_data_item_ is never read by the query path
    o.write((const char *) zero.data(), (std::streamsize) (sizeof(float) * ni * vd));
}

// reg: [n_user][7] = a, b, mu, sigma, err, smax, smin -> the NormalLinearRegressionLP file layout
// (NormalLinearRegressionLP.hpp:433-443).
void write_regression_index(const std::string &dir, const char *ds, int64_t n_user, int64_t n_item,
                            const int32_t *reg_rank, int32_t S, const float *reg, int32_t nsq, int32_t stopk) {
    char path[512];
    std::snprintf(path, sizeof path,
                  "%s/memory_index/NormalLinearRegressionLP-QS-%s-n_sample_%d-n_sample_query_%d-sample_topk_%d.index",
                  dir.c_str(), ds, S, nsq, stopk);
    std::ofstream o(path, std::ios::binary);
    size_t ni = (size_t) n_item, nu = (size_t) n_user;
    int s = S;
    o.write((char *) &ni, sizeof ni); o.write((char *) &nu, sizeof nu); o.write((char *) &s, sizeof s);
    o.write((const char *) reg_rank, (std::streamsize) (sizeof(int) * (size_t) S));
    std::vector<float> ab(2 * nu), ms(2 * nu), er(nu), ex(2 * nu);
    for (size_t u = 0; u < nu; u++) {
        ab[2 * u] = reg[7 * u]; ab[2 * u + 1] = reg[7 * u + 1];
        ms[2 * u] = reg[7 * u + 2]; ms[2 * u + 1] = reg[7 * u + 3];
        er[u] = reg[7 * u + 4];
        ex[2 * u] = reg[7 * u + 5]; ex[2 * u + 1] = reg[7 * u + 6];
    }
    o.write((char *) ab.data(), (std::streamsize) (sizeof(float) * 2 * nu));
    o.write((char *) ms.data(), (std::streamsize) (sizeof(float) * 2 * nu));
    o.write((char *) er.data(), (std::streamsize) (sizeof(float) * nu));
    o.write((char *) ex.data(), (std::streamsize) (sizeof(float) * 2 * nu));
}

struct RefUserRank { int32_t user_id, rank; float query_ip; };
struct RefStats { int32_t n_prune, n_result, n_refine, n_candidate; int64_t n_compute_item, ip_cost; };

void copy_results(const std::vector<std::vector<UserRankElement>> &res, const std::vector<SingleQueryPerformance> &perf,
                  int32_t topk, RefUserRank *out, RefStats *st) {
    for (size_t q = 0; q < res.size(); q++) {
        for (int32_t k = 0; k < topk; k++) {
            out[q * topk + k].user_id = res[q][k].userID_;
            out[q * topk + k].rank = res[q][k].rank_;
            out[q * topk + k].query_ip = res[q][k].queryIP_;
        }
        if (st) {
            st[q].n_prune = perf[q].n_prune_user_;
            st[q].n_result = perf[q].n_result_user_;
            st[q].n_refine = perf[q].n_refine_user_;
            st[q].n_candidate = 0;
            st[q].n_compute_item = 0;
            st[q].ip_cost = (int64_t) perf[q].ip_cost_;
        }
    }
}

}  // namespace

extern "C" {

int ref_set_threads(int n) { omp_set_num_threads(n); return omp_get_max_threads(); }

float ref_inner_product(const float *a, const float *b, int32_t d) { return InnerProduct(a, b, d); }

// VectorMatrix::vectorNormalize (VectorMatrix.hpp:51-66), in place.
int ref_normalize(float *v, int64_t n, int32_t d) {
    VectorMatrix vm;
    fill_vm(vm, v, n, d);
    vm.vectorNormalize();
    std::memcpy(v, vm.getRawData(), sizeof(float) * (size_t) n * (size_t) d);
    return 0;
}

// ComputeScoreTableBatch (CPU path) rows for users [start, start + n): sorted descending.
int ref_score_sort_rows(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                        int64_t start, int64_t n_rows, float *rows_out) {
    VectorMatrix u, it;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    ComputeScoreTableBatch cstb(u, it);
    cstb.ComputeSortItemsBatch((int) start, (int) n_rows, rows_out);
    return 0;
}

// bsibc: BuildSampleIndexByComputation.cpp:66-154 with an in-memory rank list; thresholds out.
int ref_build_thresholds(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                         const int32_t *sample_rank, int32_t S, float *thr_out) {
    VectorMatrix u, it;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    std::vector<int> rank_l(sample_rank, sample_rank + S);
    SampleSearch ss((int) n_item, (int) n_user, rank_l, S);
    ComputeScoreTableBatch cstb(u, it);
    const int64_t batch = 64;
    std::vector<float> rows((size_t) (batch * n_item));
    for (int64_t start = 0; start < n_user; start += batch) {
        const int64_t nb = std::min(batch, n_user - start);
        cstb.ComputeSortItemsBatch((int) start, (int) nb, rows.data());
        for (int64_t b = 0; b < nb; b++) ss.LoopPreprocess(rows.data() + b * n_item, (int) (start + b));
    }
    for (int64_t uu = 0; uu < n_user; uu++) std::memcpy(thr_out + uu * S, ss.SampleData((int) uu), sizeof(float) * S);
    return 0;
}

// SampleItem (QueryRankBySample.hpp:20-37): the mt19937(0) shuffle of the item ids.
int ref_sample_item(int32_t n_item, int32_t n_sample_item, int32_t *out) {
    std::vector<int> l(n_sample_item);
    SampleItem(n_item, n_sample_item, l);
    std::memcpy(out, l.data(), sizeof(int) * (size_t) n_sample_item);
    return 0;
}

// qdibc core: ComputeQueryRankByComputation (QueryRankByComputation.hpp:122-242), accumulated
// histogram in sampled-item order ([n_sample_item][n_item + 1]).
int ref_query_rank_distribution(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                                const int32_t *sample_item, int32_t n_sample_item, int32_t *accu_out) {
    VectorMatrix u, it;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    std::vector<int> ids(sample_item, sample_item + n_sample_item);
    std::vector<int> accu((size_t) n_sample_item * (size_t) (n_item + 1));
    double t0, t1, t2, t3;
    ComputeQueryRankByComputation(u, it, ids, n_sample_item, accu, t0, t1, t2, t3);
    std::memcpy(accu_out, accu.data(), sizeof(int) * accu.size());
    return 0;
}

// ComputeSortKthRank (QueryRankBySample.hpp:103-134).
int ref_sort_kth_rank(const int32_t *accu, int64_t n_item, int32_t n_sample_item, int32_t sample_topk,
                      int32_t *sort_kth_out, int32_t *sort_sample_id_out) {
    std::vector<int> a(accu, accu + (size_t) n_sample_item * (size_t) (n_item + 1));
    std::vector<int> kth(n_sample_item), sid(n_sample_item);
    ComputeSortKthRank(a, (int) n_item, n_sample_item, sample_topk, kth, sid);
    std::memcpy(sort_kth_out, kth.data(), sizeof(int) * (size_t) n_sample_item);
    std::memcpy(sort_sample_id_out, sid.data(), sizeof(int) * (size_t) n_sample_item);
    return 0;
}

// qdibc file output + fsr: WriteDistributionBelowTopk (build-index/FileIO.hpp:114-196) into
// work_dir, then FindOptimalSampleFast (OptimalSampleRankFast.hpp:269-472) reading it back.
int ref_find_optimal_sample_rank(const char *work_dir, int64_t n_user, int64_t n_item, int32_t n_sample,
                                 const int32_t *sample_item, const int32_t *accu, int32_t n_sample_item,
                                 int32_t sample_topk, int32_t *out, int64_t *train_cost) {
    const std::string dir(work_dir);
    ensure_index_dirs(dir);
    std::vector<int> a(accu, accu + (size_t) n_sample_item * (size_t) (n_item + 1));
    std::vector<int> kth(n_sample_item), sid(n_sample_item), ids(sample_item, sample_item + n_sample_item);
    ComputeSortKthRank(a, (int) n_item, n_sample_item, sample_topk, kth, sid);
    WriteDistributionBelowTopk(ids, kth, sid, a, n_item, n_sample_item, sample_topk, "h", dir.c_str());
    std::vector<int> rank_l(n_sample);
    size_t cost = 0;
    FindOptimalSampleFast(n_user, n_item, n_sample, rank_l, n_sample_item, sample_topk, "h", "OptimalPart",
                          dir.c_str(), cost);
    std::memcpy(out, rank_l.data(), sizeof(int) * (size_t) n_sample);
    if (train_cost) *train_cost = (int64_t) cost;
    return 0;
}

int ref_uniform_sample_rank(int32_t n_item, int32_t n_sample, int32_t *out) {
    std::vector<int> l(n_sample);
    FindUniformSample(n_item, n_sample, l);
    std::memcpy(out, l.data(), sizeof(int) * (size_t) n_sample);
    return 0;
}

// bri: NormalLinearRegressionLP fit (StartPreprocess / BatchLoopPreprocess / SaveIndex) over the
// given thresholds; the saved file is read back into rec_out [n_user][7].
int ref_fit_regression(const char *work_dir, const float *thr, int64_t n_user, int64_t n_item,
                       const int32_t *sample_rank, int32_t S, float *rec_out) {
    const std::string dir(work_dir);
    ensure_index_dirs(dir);
    NormalLinearRegressionLP lr((int) n_item, (int) n_user, "QS");
    lr.StartPreprocess(sample_rank, S);
    const int bn = BaseLinearRegression::batch_n_user_;
    for (int64_t start = 0; start < n_user; start += bn) {
        const int np = (int) std::min<int64_t>(bn, n_user - start);
        std::vector<const float *> l(np);
        for (int i = 0; i < np; i++) l[i] = thr + (start + i) * S;
        double t0, t1, t2;
        lr.BatchLoopPreprocess(l, (int) start, np, t0, t1, t2);
    }
    lr.FinishPreprocess();
    lr.SaveIndex(dir.c_str(), "h", 0, 0);
    char path[512];
    std::snprintf(path, sizeof path,
                  "%s/memory_index/NormalLinearRegressionLP-QS-h-n_sample_%d-n_sample_query_0-sample_topk_0.index",
                  dir.c_str(), S);
    std::ifstream in(path, std::ios::binary);
    if (!in) return -1;
    size_t ni, nu; int s;
    in.read((char *) &ni, sizeof ni); in.read((char *) &nu, sizeof nu); in.read((char *) &s, sizeof s);
    std::vector<int> rk(s);
    in.read((char *) rk.data(), sizeof(int) * (size_t) s);
    std::vector<float> ab(2 * nu), ms(2 * nu), er(nu), ex(2 * nu);
    in.read((char *) ab.data(), sizeof(float) * 2 * nu);
    in.read((char *) ms.data(), sizeof(float) * 2 * nu);
    in.read((char *) er.data(), sizeof(float) * nu);
    in.read((char *) ex.data(), sizeof(float) * 2 * nu);
    for (size_t u = 0; u < nu; u++) {
        float *r = rec_out + 7 * u;
        r[0] = ab[2 * u]; r[1] = ab[2 * u + 1]; r[2] = ms[2 * u]; r[3] = ms[2 * u + 1];
        r[4] = er[u]; r[5] = ex[2 * u]; r[6] = ex[2 * u + 1];
    }
    return 0;
}

// NormalLinearRegressionLP::ComputeRankBound for one user, loading the model the reference way.
int ref_regression_rank_bound(const char *work_dir, int64_t n_user, int64_t n_item, const int32_t *reg_rank,
                              int32_t S, const float *reg, int64_t n_eval, const int32_t *user_ids,
                              const float *qlb, const float *qub, int32_t *lb_out, int32_t *ub_out) {
    const std::string dir(work_dir);
    ensure_index_dirs(dir);
    write_regression_index(dir, "h", n_user, n_item, reg_rank, S, reg, 0, 0);
    NormalLinearRegressionLP lr(dir.c_str(), "h", "QS", S, 0, 0, 1);
    for (int64_t i = 0; i < n_eval; i++) {
        int l, u;
        lr.ComputeRankBound(qlb[i], qub[i], user_ids[i], l, u);
        lb_out[i] = l; ub_out[i] = u;
    }
    return 0;
}

// bsibc / fsr: a SampleSearch index file written by SampleSearch::SaveIndex (SampleSearch.hpp:158-197)
// under work_dir/memory_index, named as the reference names it.
int ref_write_sample_search(const char *work_dir, const char *ds, const char *name, const int32_t *rank, int32_t S,
                            const float *thr, int64_t n_user, int64_t n_item, int32_t nsq, int32_t stopk,
                            int32_t is_query_distribution) {
    ensure_index_dirs(work_dir);
    write_sample_index(work_dir, ds, name, rank, S, thr, n_user, n_item, nsq, stopk, is_query_distribution != 0);
    return 0;
}

// qdibc: the query-distribution directory written by WriteDistributionBelowTopk
// (src/app/build-index/FileIO.hpp:57-137) under work_dir/query_distribution.
int ref_write_query_distribution(const char *work_dir, const char *ds, const int32_t *sample_item,
                                 const int32_t *sort_kth, const int32_t *sort_sid, const int32_t *accu, int64_t n_item,
                                 int32_t n_sample_item, int32_t sample_topk) {
    ensure_index_dirs(work_dir);
    const size_t n = (size_t) n_sample_item;
    std::vector<int> si(sample_item, sample_item + n), sk(sort_kth, sort_kth + n), sid(sort_sid, sort_sid + n);
    std::vector<int> acc(accu, accu + n * (size_t) (n_item + 1));
    WriteDistributionBelowTopk(si, sk, sid, acc, n_item, n_sample_item, sample_topk, ds, work_dir);
    return 0;
}

// bsvdi: SVD(user, item, SIGMA) (SVD.hpp:62-124; the decomposition itself is the stand-in's).
int ref_svd_build(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d, float sigma,
                  float *transfer_item_out, float *svd_user_out, int32_t *check_dim_out) {
    VectorMatrix u, it;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    SVD svd(u, it, sigma);
    std::memcpy(transfer_item_out, svd.transfer_item_.getRawData(), sizeof(float) * (size_t) d * (size_t) d);
    std::memcpy(svd_user_out, svd.transfer_user_.getRawData(), sizeof(float) * (size_t) n_user * (size_t) d);
    *check_dim_out = svd.check_dim_;
    return 0;
}

// QS::Index::Retrieval (QS.hpp:106-230) on an index written to work_dir in the reference formats.
int ref_qs_retrieval(const char *work_dir, const float *user, int64_t n_user, const float *item, int64_t n_item,
                     int32_t d, int32_t check_dim, const int32_t *sample_rank, int32_t S, const float *thr,
                     const float *query, int32_t n_query, int32_t topk, int32_t n_thread,
                     RefUserRank *out, RefStats *st) {
    const std::string dir(work_dir);
    ensure_index_dirs(dir);
    write_sample_index(dir, "h", "QS", sample_rank, S, thr, n_user, n_item, 0, 0, true);
    VectorMatrix u, it, qv;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    fill_vm(qv, query, n_query, d);
    SampleSearch rank_ins(dir.c_str(), "h", "QS", S, true, true, 0, 0, n_thread);
    ComputeAllIPBound disk_ins(u, it, check_dim, n_thread);
    QS::Index idx(rank_ins, disk_ins, u, (int) n_user, (int) n_item, d, n_thread);
    std::vector<SingleQueryPerformance> perf(n_query);
    auto res = idx.Retrieval(qv, topk, n_query, perf);
    copy_results(res, perf, topk, out, st);
    return 0;
}

// US::Index::Retrieval (US.hpp:96-213).  Returns the number of queries answered.
int ref_us_retrieval(const char *work_dir, const float *user, int64_t n_user, const float *item, int64_t n_item,
                     int32_t d, const int32_t *sample_rank, int32_t S, const float *thr,
                     const float *query, int32_t n_query, int32_t topk, int32_t n_thread,
                     RefUserRank *out, RefStats *st) {
    const std::string dir(work_dir);
    ensure_index_dirs(dir);
    write_sample_index(dir, "h", "US", sample_rank, S, thr, n_user, n_item, 0, 0, false);
    VectorMatrix u, it, qv;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    fill_vm(qv, query, n_query, d);
    auto idx = US::BuildIndex(it, u, "h", dir.c_str(), S, n_thread);
    const int nq = S <= 1000 ? 100 : n_query;
    std::vector<SingleQueryPerformance> perf(nq);
    auto res = idx->Retrieval(qv, topk, n_query, perf);
    copy_results(res, perf, topk, out, st);
    return nq;
}

// QSRPNormalLP::BuildIndex + Retrieval (QSRPNormalLP.hpp:116-323) on an index written to work_dir.
int ref_qsrp_retrieval(const char *work_dir, const float *user, const float *svd_user, const float *transfer_item,
                       int64_t n_user, const float *item, int64_t n_item, int32_t d, int32_t check_dim,
                       const int32_t *sample_rank, int32_t S, const float *thr,
                       const int32_t *reg_rank, const float *reg,
                       const float *query, int32_t n_query, int32_t topk, int32_t n_thread,
                       RefUserRank *out, RefStats *st) {
    const std::string dir(work_dir);
    ensure_index_dirs(dir);
    write_sample_index(dir, "h", "QS", sample_rank, S, thr, n_user, n_item, 1, 1, true);
    write_svd_index(dir, "h", n_user, n_item, d, check_dim, transfer_item, svd_user);
    write_regression_index(dir, "h", n_user, n_item, reg_rank, S, reg, 1, 1);
    VectorMatrix u, it, qv;
    fill_vm(u, user, n_user, d);
    fill_vm(it, item, n_item, d);
    fill_vm(qv, query, n_query, d);
    auto idx = QSRPNormalLP::BuildIndex(it, u, "h", S, 1, 1, n_thread, dir.c_str());
    std::vector<SingleQueryPerformance> perf(n_query);
    auto res = idx->Retrieval(qv, topk, n_query, perf);
    copy_results(res, perf, topk, out, st);
    return 0;
}

}  // extern "C"

extern "C" {
// NormalLinearRegressionLP::CDFPhi (NormalLinearRegressionLP.hpp:123-143) over an array.
int ref_cdf_phi(const float *x, int64_t n, float *out) {
    NormalLinearRegressionLP lr(1, 1, "QS");
    for (int64_t i = 0; i < n; i++) out[i] = lr.CDFPhi(x[i]);
    return 0;
}
}

// ---- persistent reference index for timing (bench.py's CPU legs) --------------------------------
namespace {
struct RefQsrp {
    std::string dir;
    VectorMatrix user, item;
    std::unique_ptr<QSRPNormalLP::Index> idx;
    int64_t n_user = 0;
    int32_t dim = 0;
};
}  // namespace

extern "C" {
// QSRPNormalLP::BuildIndex from index files written to work_dir in the reference formats; the
// handle keeps the reference's Index object for repeated Retrieval calls.
void *ref_qsrp_open(const char *work_dir, const float *user, const float *svd_user, const float *transfer_item,
                    int64_t n_user, const float *item, int64_t n_item, int32_t d, int32_t check_dim,
                    const int32_t *sample_rank, int32_t S, const float *thr, const int32_t *reg_rank, const float *reg,
                    int32_t n_thread) {
    RefQsrp *h = new RefQsrp();
    h->dir = work_dir;
    ensure_index_dirs(h->dir);
    write_sample_index(h->dir, "h", "QS", sample_rank, S, thr, n_user, n_item, 1, 1, true);
    write_svd_index(h->dir, "h", n_user, n_item, d, check_dim, transfer_item, svd_user);
    write_regression_index(h->dir, "h", n_user, n_item, reg_rank, S, reg, 1, 1);
    fill_vm(h->user, user, n_user, d);
    fill_vm(h->item, item, n_item, d);
    h->idx = QSRPNormalLP::BuildIndex(h->item, h->user, "h", S, 1, 1, n_thread, h->dir.c_str());
    h->n_user = n_user;
    h->dim = d;
    return h;
}

// Index::Retrieval on n_query queries; *seconds = wall time of the Retrieval call alone.
int ref_qsrp_run(void *handle, const float *query, int32_t n_query, int32_t topk, RefUserRank *out, RefStats *st,
                 double *seconds) {
    RefQsrp *h = static_cast<RefQsrp *>(handle);
    VectorMatrix qv;
    fill_vm(qv, query, n_query, h->dim);
    std::vector<SingleQueryPerformance> perf(n_query);
    const auto t0 = std::chrono::steady_clock::now();
    auto res = h->idx->Retrieval(qv, topk, n_query, perf);
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (out) copy_results(res, perf, topk, out, st);
    return 0;
}

void ref_qsrp_close(void *handle) {
    RefQsrp *h = static_cast<RefQsrp *>(handle);
    std::filesystem::remove_all(h->dir);
    delete h;
}
}
