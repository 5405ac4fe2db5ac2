// rri_b200 -- TEST INFRASTRUCTURE: the reference's query app run two ways on one set of index files.
//
// Loads a dataset with the reference's readData (util/VectorIO.hpp:39-68), builds the reference's
// own index of the method from the index files (QS::BuildIndex, QSRPNormalLP::BuildIndex,
// US::BuildIndex, as src/app/ReverseRankIndex.cpp:105-172 does) and the B200 mirror of it
// (reverse-k-ranks_b200/host/B200Index.hpp, librkr_b200 through include/rkr.h), answers the query
// file with each, and writes both result sets through the reference's WriteRankResult
// (util/FileIO.hpp:83-148) as <dataset>-<method>-ref-* and <dataset>-<method>-b200-* under
// ../result/rank (the reference's relative layout: run it from a directory whose sibling is
// result/rank).  A test compares the two sets of CSV files byte for byte.
//
// usage: rri_b200 dataset_dir dataset_name index_dir method topk n_sample n_sample_query sample_topk
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

#include "util/VectorIO.hpp"
#include "util/TimeMemory.hpp"
#include "util/FileIO.hpp"
#include "struct/UserRankElement.hpp"
#include "struct/VectorMatrix.hpp"
#include "QS.hpp"
#include "QSRPNormalLP.hpp"
#include "US.hpp"
#include "B200Index.hpp"

using namespace ReverseMIPS;

int main(int argc, char **argv) {
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s dataset_dir dataset_name index_dir method topk n_sample n_sample_query "
                             "sample_topk\n", argv[0]);
        return 2;
    }
    const char *dataset_dir = argv[1], *ds = argv[2], *index_dir = argv[3];
    const std::string method = argv[4];
    const int topk = std::atoi(argv[5]), n_sample = std::atoi(argv[6]), nsq = std::atoi(argv[7]),
              stopk = std::atoi(argv[8]);
    int n_item = 0, n_query = 0, n_user = 0, dim = 0;
    std::vector<VectorMatrix> data = readData(dataset_dir, ds, n_item, n_query, n_user, dim);
    VectorMatrix &user = data[0], &item = data[1], &query = data[2];
    try {
        // the mirror first: the reference's factories take the user matrix by reference
        std::unique_ptr<BaseIndex> b200 = B200::BuildIndex(method, item, user, ds, n_sample, nsq, stopk, index_dir);
        std::vector<SingleQueryPerformance> perf_b(n_query);
        auto res_b = b200->Retrieval(query, topk, n_query, perf_b);
        std::unique_ptr<BaseIndex> ref;
        if (method == "QS") ref = QS::BuildIndex(item, user, ds, n_sample, nsq, stopk, 1, index_dir);
        else if (method == "QSRPNormalLP") ref = QSRPNormalLP::BuildIndex(item, user, ds, n_sample, nsq, stopk, 1, index_dir);
        else if (method == "US") ref = US::BuildIndex(item, user, ds, index_dir, n_sample, 1);
        else throw std::runtime_error("unknown method " + method);
        std::vector<SingleQueryPerformance> perf_r(n_query);
        auto res_r = ref->Retrieval(query, topk, n_query, perf_r);
        WriteRankResult(res_r, ds, method.c_str(), "ref");
        WriteRankResult(res_b, ds, method.c_str(), "b200");
        std::printf("%s: %zu / %zu queries answered\n", method.c_str(), res_r.size(), res_b.size());
    } catch (const std::exception &e) {
        std::fprintf(stderr, "rri_b200: %s\n", e.what());
        return 1;
    }
    return 0;
}
