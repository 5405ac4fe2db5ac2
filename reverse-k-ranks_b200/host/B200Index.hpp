// B200Index.hpp -- a BaseIndex for the reference's query app (src/app/ReverseRankIndex.cpp) that
// answers QS / QSRPNormalLP / US retrieval on a B200 through librkr_b200's C ABI (include/rkr.h).
//
// Header-only C++ meant to be compiled inside the reference's build (it uses the reference's
// VectorMatrix, UserRankElement and SingleQueryPerformance types; the library reads the reference's
// own index files), linked with -lrkr_b200.  It mirrors the reference's factories
// (QS::BuildIndex, src/impl/QS.hpp:259-288; QSRPNormalLP::BuildIndex, src/impl/QSRPNormalLP.hpp:289-323;
// US::BuildIndex, src/impl/US.hpp:226-242) and Index::Retrieval; errors throw std::runtime_error
// where the reference would log and exit.
#ifndef RKR_B200_INDEX_HPP
#define RKR_B200_INDEX_HPP

#include <chrono>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "rkr.h"

namespace ReverseMIPS::B200 {

inline void check(int status, const char *what) {
    if (status != RKR_OK) throw std::runtime_error(std::string(what) + ": " + rkr_last_error());
}

class Index : public BaseIndex {
    rkr_index *h_ = nullptr;
    int method_ = RKR_METHOD_QS;
    int n_user_ = 0;
    double total_time_ = 0;
    int64_t total_refine_user_ = 0, total_ip_cost_ = 0;

public:
    Index(rkr_index *h, int method, int n_user) : h_(h), method_(method), n_user_(n_user) {}
    ~Index() override { rkr_index_destroy(h_); }
    Index(const Index &) = delete;
    Index &operator=(const Index &) = delete;

    std::vector<std::vector<UserRankElement>> Retrieval(const VectorMatrix &query_item, const int &topk,
                                                        const int &n_execute_query,
                                                        std::vector<SingleQueryPerformance> &query_performance_l) override {
        if (n_execute_query > query_item.n_vector_) throw std::runtime_error("n_execute_query larger than n_query_item");
        if (topk > n_user_) throw std::runtime_error("top-k is too large");
        std::vector<rkr_user_rank> out((size_t) std::max(n_execute_query, 100) * topk);
        std::vector<rkr_query_stats> st((size_t) std::max(n_execute_query, 100));
        int32_t n_answered = 0;
        const auto t0 = std::chrono::steady_clock::now();
        check(rkr_retrieval(h_, method_, query_item.getRawData(), n_execute_query, topk, out.data(), st.data(),
                            &n_answered),
              "rkr_retrieval");
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        total_time_ += secs;
        std::vector<std::vector<UserRankElement>> res(n_answered, std::vector<UserRankElement>(topk));
        if ((int) query_performance_l.size() < n_answered) query_performance_l.resize(n_answered);
        for (int q = 0; q < n_answered; q++) {
            for (int k = 0; k < topk; k++) {
                const rkr_user_rank &e = out[(size_t) q * topk + k];
                res[q][k] = UserRankElement(e.user_id, e.rank, e.query_ip);
            }
            total_refine_user_ += st[q].n_refine;
            total_ip_cost_ += st[q].ip_cost;
            query_performance_l[q] = SingleQueryPerformance(q, st[q].n_prune, st[q].n_result, st[q].n_refine,
                                                            (size_t) st[q].ip_cost, 0, secs / n_answered, 0, 0);
        }
        return res;
    }

    std::string PerformanceStatistics(const int &topk) override {
        char buff[512];
        std::snprintf(buff, sizeof buff, "top%d retrieval time: total %.3fs (B200)\n\ttotal ip cost %lld, total refine user %lld",
                      topk, total_time_, (long long) total_ip_cost_, (long long) total_refine_user_);
        return buff;
    }

    uint64_t IndexSizeByte() override {
        uint64_t b = 0;
        check(rkr_index_size_bytes(h_, &b), "rkr_index_size_bytes");
        return b;
    }
};

// method: "QS", "QSRPNormalLP" or "US"; the index files are the ones fsr/bsibc/bri/bsvdi wrote.
inline std::unique_ptr<Index> BuildIndex(const std::string &method, const VectorMatrix &data_item,
                                         const VectorMatrix &user, const char *dataset_name, int n_sample,
                                         int n_sample_query, int sample_topk, const char *index_dir,
                                         int device = 0) {
    const int m = method == "QS" ? RKR_METHOD_QS
                  : method == "QSRPNormalLP" ? RKR_METHOD_QSRP_NORMAL_LP
                  : method == "US" ? RKR_METHOD_US : -1;
    if (m < 0) throw std::runtime_error("not such method");
    rkr_index *h = nullptr;
    check(rkr_index_create(device, user.getRawData(), user.n_vector_, data_item.getRawData(), data_item.n_vector_,
                           user.vec_dim_, &h),
          "rkr_index_create");
    std::unique_ptr<Index> idx = std::make_unique<Index>(h, m, user.n_vector_);
    // the files the reference's factory reads: the SampleSearch index (SampleSearch::LoadIndex,
    // SampleSearch.hpp:199-244), the SVD index (SVD::LoadIndex, SVD.hpp:154-188) and the regression
    // index (NormalLinearRegressionLP::LoadIndex, NormalLinearRegressionLP.hpp:448-487), read by the
    // library from memory maps
    check(rkr_index_load_files(h, m, index_dir, dataset_name, n_sample, n_sample_query, sample_topk),
          "rkr_index_load_files");
    return idx;
}

}  // namespace ReverseMIPS::B200

#endif  // RKR_B200_INDEX_HPP
