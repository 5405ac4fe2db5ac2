// rkr_files.cpp -- the reference's on-disk index formats, read and written natively.
//
// The reference's build apps hand their results to the query app through files: the SampleSearch
// index (SampleSearch::SaveIndex / LoadIndex, SampleSearch.hpp:158-244), the NormalLinearRegressionLP
// index (NormalLinearRegressionLP.hpp:419-487), the SVD index (SVD.hpp:126-188) and the query
// distribution directory (WriteDistributionBelowTopk, src/app/build-index/FileIO.hpp:57-137;
// ReadQueryDistribution, OptimalSampleRank.hpp:157-200).  This file reads and writes the same bytes
// (native-endian size_t / int / float, no padding), so the engine's build steps and the reference's
// apps can take each other's files, and loads a method's whole file set into an index from memory
// maps of the files (rkr_index_load_files).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rkr.h"

namespace rkr {
void set_error(const char *fmt, ...);
}

namespace {

using rkr::set_error;

// A read-only memory map of a whole file.
struct Mapped {
    const unsigned char *p = nullptr;
    size_t n = 0;
    int open(const char *path) {
        const int fd = ::open(path, O_RDONLY);
        if (fd < 0) {
            set_error("cannot open %s: %s", path, std::strerror(errno));
            return RKR_ERR_IO;
        }
        struct stat st {};
        if (fstat(fd, &st) != 0) {
            set_error("cannot stat %s: %s", path, std::strerror(errno));
            ::close(fd);
            return RKR_ERR_IO;
        }
        n = (size_t) st.st_size;
        if (n) {
            void *m = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m == MAP_FAILED) {
                set_error("cannot map %s: %s", path, std::strerror(errno));
                ::close(fd);
                return RKR_ERR_IO;
            }
            p = static_cast<const unsigned char *>(m);
        }
        ::close(fd);
        return RKR_OK;
    }
    ~Mapped() {
        if (p) munmap(const_cast<unsigned char *>(p), n);
    }
    template <class T>
    T at(size_t off) const {
        T v;
        std::memcpy(&v, p + off, sizeof v);
        return v;
    }
};

// Sequential writer; every failure is reported once, at close.
struct Writer {
    FILE *f = nullptr;
    bool ok = true;
    std::string path;
    int open(const char *p) {
        path = p;
        f = std::fopen(p, "wb");
        if (!f) {
            set_error("cannot create %s: %s", p, std::strerror(errno));
            return RKR_ERR_IO;
        }
        return RKR_OK;
    }
    void put(const void *d, size_t n) {
        if (ok && n && std::fwrite(d, 1, n, f) != n) ok = false;
    }
    template <class T>
    void val(T v) { put(&v, sizeof v); }
    int close() {
        const bool c = std::fclose(f) == 0;
        f = nullptr;
        if (!ok || !c) {
            set_error("write to %s failed", path.c_str());
            return RKR_ERR_IO;
        }
        return RKR_OK;
    }
    ~Writer() {
        if (f) std::fclose(f);
    }
};

// SampleSearch layout: size_t n_sample, n_item, n_user; int rank[n_sample]; optionally
// float thresholds[n_user][n_sample] (the memory_index form; the qrs_to_sample_index form stops
// after the ranks).
struct SampleSearchView {
    int64_t n_sample = 0, n_item = 0, n_user = 0;
    const int32_t *rank = nullptr;
    const float *thr = nullptr;
    int parse(const Mapped &m, const char *path) {
        if (m.n < 24) {
            set_error("%s: shorter than the SampleSearch header", path);
            return RKR_ERR_IO;
        }
        const uint64_t s = m.at<uint64_t>(0), ni = m.at<uint64_t>(8), nu = m.at<uint64_t>(16);
        if (s == 0 || s > (1u << 20) || ni > (1ull << 40) || nu > (1ull << 40) || m.n < 24 + 4 * s) {
            set_error("%s: not a SampleSearch index (n_sample %llu, n_item %llu, n_user %llu, %zu bytes)", path,
                      (unsigned long long) s, (unsigned long long) ni, (unsigned long long) nu, m.n);
            return RKR_ERR_IO;
        }
        n_sample = (int64_t) s, n_item = (int64_t) ni, n_user = (int64_t) nu;
        rank = reinterpret_cast<const int32_t *>(m.p + 24);
        const size_t full = 24 + 4 * s + 4 * s * nu;
        if (m.n == full) thr = reinterpret_cast<const float *>(m.p + 24 + 4 * s);
        else if (m.n != 24 + 4 * s) {
            set_error("%s: %zu bytes, expected %zu (with scores) or %zu (ranks only)", path, m.n, full,
                      (size_t) (24 + 4 * s));
            return RKR_ERR_IO;
        }
        return RKR_OK;
    }
};

// NormalLinearRegressionLP layout: size_t n_item, n_user; int n_sample; int rank[n_sample];
// float (a, b)[n_user], (mu, sigma)[n_user], err[n_user], (smax, smin)[n_user].
struct RegressionView {
    int64_t n_item = 0, n_user = 0;
    int32_t n_sample = 0;
    const int32_t *rank = nullptr;
    const float *ab = nullptr, *ms = nullptr, *er = nullptr, *ex = nullptr;
    int parse(const Mapped &m, const char *path) {
        if (m.n < 20) {
            set_error("%s: shorter than the regression header", path);
            return RKR_ERR_IO;
        }
        const uint64_t ni = m.at<uint64_t>(0), nu = m.at<uint64_t>(8);
        const int32_t s = m.at<int32_t>(16);
        if (s <= 0 || s > (1 << 20) || nu > (1ull << 40) || ni > (1ull << 40) ||
            m.n != 20 + 4 * (size_t) s + 28 * nu) {
            set_error("%s: not a NormalLinearRegressionLP index (n_sample %d, n_user %llu, %zu bytes)", path, s,
                      (unsigned long long) nu, m.n);
            return RKR_ERR_IO;
        }
        n_item = (int64_t) ni, n_user = (int64_t) nu, n_sample = s;
        rank = reinterpret_cast<const int32_t *>(m.p + 20);
        const float *f = reinterpret_cast<const float *>(m.p + 20 + 4 * (size_t) s);
        ab = f, ms = f + 2 * nu, er = f + 4 * nu, ex = f + 5 * nu;
        return RKR_OK;
    }
    void records(float *out) const {  // -> [n_user][7] a, b, mu, sigma, err, smax, smin
        for (int64_t u = 0; u < n_user; u++) {
            float *r = out + 7 * u;
            r[0] = ab[2 * u], r[1] = ab[2 * u + 1], r[2] = ms[2 * u], r[3] = ms[2 * u + 1];
            r[4] = er[u], r[5] = ex[2 * u], r[6] = ex[2 * u + 1];
        }
    }
};

// SVD layout: size_t n_user, n_item, dim; float sigma; int check_dim; float transfer_item[dim][dim],
// svd_user[n_user][dim], svd_item[n_item][dim].
struct SvdView {
    int64_t n_user = 0, n_item = 0;
    int32_t dim = 0, check_dim = 0;
    float sigma = 0.0f;
    const float *transfer = nullptr, *user = nullptr, *item = nullptr;
    int parse(const Mapped &m, const char *path) {
        if (m.n < 32) {
            set_error("%s: shorter than the SVD header", path);
            return RKR_ERR_IO;
        }
        const uint64_t nu = m.at<uint64_t>(0), ni = m.at<uint64_t>(8), d = m.at<uint64_t>(16);
        const float sg = m.at<float>(24);
        const int32_t cd = m.at<int32_t>(28);
        if (d == 0 || d > 4096 || nu > (1ull << 40) || ni > (1ull << 40) || cd < 0 || (uint64_t) cd > d ||
            m.n != 32 + 4 * d * (d + nu + ni)) {
            set_error("%s: not an SVD index (dim %llu, n_user %llu, n_item %llu, %zu bytes)", path,
                      (unsigned long long) d, (unsigned long long) nu, (unsigned long long) ni, m.n);
            return RKR_ERR_IO;
        }
        n_user = (int64_t) nu, n_item = (int64_t) ni, dim = (int32_t) d, sigma = sg, check_dim = cd;
        transfer = reinterpret_cast<const float *>(m.p + 32);
        user = transfer + d * d;
        item = user + nu * d;
        return RKR_OK;
    }
};

std::string fmt(const char *f, ...) __attribute__((format(printf, 1, 2)));
std::string fmt(const char *f, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    std::vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

}  // namespace

extern "C" {

int rkr_file_sample_search_info(const char *path, int32_t *n_sample, int64_t *n_item, int64_t *n_user,
                                int32_t *has_scores) {
    if (!path) {
        set_error("null path");
        return RKR_ERR_INVALID;
    }
    Mapped m;
    SampleSearchView v;
    int st = m.open(path);
    if (st == RKR_OK) st = v.parse(m, path);
    if (st != RKR_OK) return st;
    if (n_sample) *n_sample = (int32_t) v.n_sample;
    if (n_item) *n_item = v.n_item;
    if (n_user) *n_user = v.n_user;
    if (has_scores) *has_scores = v.thr != nullptr;
    return RKR_OK;
}

int rkr_file_read_sample_search(const char *path, int32_t *rank_out, float *thresholds_out) {
    if (!path) {
        set_error("null path");
        return RKR_ERR_INVALID;
    }
    Mapped m;
    SampleSearchView v;
    int st = m.open(path);
    if (st == RKR_OK) st = v.parse(m, path);
    if (st != RKR_OK) return st;
    if (rank_out) std::memcpy(rank_out, v.rank, 4 * (size_t) v.n_sample);
    if (thresholds_out) {
        if (!v.thr) {
            set_error("%s holds no thresholds (a ranks-only index)", path);
            return RKR_ERR_STATE;
        }
        std::memcpy(thresholds_out, v.thr, 4 * (size_t) v.n_sample * (size_t) v.n_user);
    }
    return RKR_OK;
}

int rkr_file_write_sample_search(const char *path, const int32_t *rank, int32_t n_sample, int64_t n_item,
                                 int64_t n_user, const float *thresholds) {
    if (!path || !rank || n_sample <= 0 || n_item < 0 || n_user < 0) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    Writer w;
    if (int st = w.open(path)) return st;
    w.val<uint64_t>((uint64_t) n_sample);
    w.val<uint64_t>((uint64_t) n_item);
    w.val<uint64_t>((uint64_t) n_user);
    w.put(rank, 4 * (size_t) n_sample);
    if (thresholds) w.put(thresholds, 4 * (size_t) n_sample * (size_t) n_user);
    return w.close();
}

int rkr_file_regression_info(const char *path, int32_t *n_sample, int64_t *n_item, int64_t *n_user) {
    if (!path) {
        set_error("null path");
        return RKR_ERR_INVALID;
    }
    Mapped m;
    RegressionView v;
    int st = m.open(path);
    if (st == RKR_OK) st = v.parse(m, path);
    if (st != RKR_OK) return st;
    if (n_sample) *n_sample = v.n_sample;
    if (n_item) *n_item = v.n_item;
    if (n_user) *n_user = v.n_user;
    return RKR_OK;
}

int rkr_file_read_regression(const char *path, int32_t *rank_out, float *records_out) {
    if (!path) {
        set_error("null path");
        return RKR_ERR_INVALID;
    }
    Mapped m;
    RegressionView v;
    int st = m.open(path);
    if (st == RKR_OK) st = v.parse(m, path);
    if (st != RKR_OK) return st;
    if (rank_out) std::memcpy(rank_out, v.rank, 4 * (size_t) v.n_sample);
    if (records_out) v.records(records_out);
    return RKR_OK;
}

int rkr_file_write_regression(const char *path, const int32_t *rank, int32_t n_sample, int64_t n_item,
                              int64_t n_user, const float *records) {
    if (!path || !rank || !records || n_sample <= 0 || n_item < 0 || n_user < 0) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    Writer w;
    if (int st = w.open(path)) return st;
    w.val<uint64_t>((uint64_t) n_item);
    w.val<uint64_t>((uint64_t) n_user);
    w.val<int32_t>(n_sample);
    w.put(rank, 4 * (size_t) n_sample);
    // the record's fields go out as the reference's four arrays, each over all users
    const int cols[4][2] = {{0, 2}, {2, 2}, {4, 1}, {5, 2}};
    std::vector<float> buf;
    for (const auto &c : cols) {
        buf.resize((size_t) n_user * c[1]);
        for (int64_t u = 0; u < n_user; u++)
            for (int j = 0; j < c[1]; j++) buf[(size_t) u * c[1] + j] = records[7 * u + c[0] + j];
        w.put(buf.data(), 4 * buf.size());
    }
    return w.close();
}

int rkr_file_svd_info(const char *path, int64_t *n_user, int64_t *n_item, int32_t *dim, float *sigma,
                      int32_t *check_dim) {
    if (!path) {
        set_error("null path");
        return RKR_ERR_INVALID;
    }
    Mapped m;
    SvdView v;
    int st = m.open(path);
    if (st == RKR_OK) st = v.parse(m, path);
    if (st != RKR_OK) return st;
    if (n_user) *n_user = v.n_user;
    if (n_item) *n_item = v.n_item;
    if (dim) *dim = v.dim;
    if (sigma) *sigma = v.sigma;
    if (check_dim) *check_dim = v.check_dim;
    return RKR_OK;
}

int rkr_file_read_svd(const char *path, float *transfer_item, float *svd_user, float *svd_item) {
    if (!path) {
        set_error("null path");
        return RKR_ERR_INVALID;
    }
    Mapped m;
    SvdView v;
    int st = m.open(path);
    if (st == RKR_OK) st = v.parse(m, path);
    if (st != RKR_OK) return st;
    const size_t d = (size_t) v.dim;
    if (transfer_item) std::memcpy(transfer_item, v.transfer, 4 * d * d);
    if (svd_user) std::memcpy(svd_user, v.user, 4 * d * (size_t) v.n_user);
    if (svd_item) std::memcpy(svd_item, v.item, 4 * d * (size_t) v.n_item);
    return RKR_OK;
}

int rkr_file_write_svd(const char *path, int64_t n_user, int64_t n_item, int32_t dim, float sigma, int32_t check_dim,
                       const float *transfer_item, const float *svd_user, const float *svd_item) {
    if (!path || !transfer_item || !svd_user || dim <= 0 || n_user < 0 || n_item < 0 || check_dim < 0 ||
        check_dim > dim) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    Writer w;
    if (int st = w.open(path)) return st;
    const size_t d = (size_t) dim;
    w.val<uint64_t>((uint64_t) n_user);
    w.val<uint64_t>((uint64_t) n_item);
    w.val<uint64_t>((uint64_t) d);
    w.val<float>(sigma);
    w.val<int32_t>(check_dim);
    w.put(transfer_item, 4 * d * d);
    w.put(svd_user, 4 * d * (size_t) n_user);
    if (svd_item) {
        w.put(svd_item, 4 * d * (size_t) n_item);
    } else {  // the query path never reads the transferred items: zeros, one row at a time
        std::vector<float> zero(d, 0.0f);
        for (int64_t i = 0; i < n_item; i++) w.put(zero.data(), 4 * d);
    }
    return w.close();
}

int rkr_file_write_query_distribution(const char *dir, const int32_t *sample_item, const int32_t *sort_kth_rank,
                                      const int32_t *sort_sample_id, const int32_t *accu, int32_t n_sample_item,
                                      int64_t n_item) {
    if (!dir || !sample_item || !sort_kth_rank || !sort_sample_id || !accu || n_sample_item <= 0 || n_item <= 0) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    if (mkdir(dir, 0755) != 0 && errno != EEXIST) {
        set_error("cannot create %s: %s", dir, std::strerror(errno));
        return RKR_ERR_IO;
    }
    for (int32_t s = 0; s < n_sample_item; s++)
        if (sort_sample_id[s] < 0 || sort_sample_id[s] >= n_sample_item) {
            set_error("sort_sample_id[%d] = %d out of range", s, sort_sample_id[s]);
            return RKR_ERR_INVALID;
        }
    {  // the sampled item ids in sorted-sample order, one decimal per line
        const std::string p = fmt("%s/sample_itemID_l.txt", dir);
        Writer w;
        if (int st = w.open(p.c_str())) return st;
        for (int32_t s = 0; s < n_sample_item; s++) {
            const std::string line = fmt("%d\n", sample_item[sort_sample_id[s]]);
            w.put(line.data(), line.size());
        }
        if (int st = w.close()) return st;
    }
    {
        const std::string p = fmt("%s/sort_kth_rank_l.index", dir);
        Writer w;
        if (int st = w.open(p.c_str())) return st;
        w.put(sort_kth_rank, 4 * (size_t) n_sample_item);
        if (int st = w.close()) return st;
    }
    const std::string p = fmt("%s/accu_n_user_rank_l.index", dir);
    Writer w;
    if (int st = w.open(p.c_str())) return st;
    for (int32_t s = 0; s < n_sample_item; s++)  // rows in sorted-sample order
        w.put(accu + (size_t) sort_sample_id[s] * (size_t) (n_item + 1), 4 * (size_t) (n_item + 1));
    return w.close();
}

int rkr_file_read_query_distribution(const char *dir, int32_t n_sample_item, int64_t n_item, int32_t *sample_item_out,
                                     int32_t *sort_kth_rank_out, int32_t *accu_out) {
    if (!dir || n_sample_item <= 0 || n_item <= 0) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    if (sample_item_out) {
        const std::string p = fmt("%s/sample_itemID_l.txt", dir);
        FILE *f = std::fopen(p.c_str(), "r");
        if (!f) {
            set_error("cannot open %s: %s", p.c_str(), std::strerror(errno));
            return RKR_ERR_IO;
        }
        int32_t s = 0;
        for (; s < n_sample_item; s++)
            if (std::fscanf(f, "%d", &sample_item_out[s]) != 1) break;
        std::fclose(f);
        if (s != n_sample_item) {
            set_error("%s: %d item ids, expected %d", p.c_str(), s, n_sample_item);
            return RKR_ERR_IO;
        }
    }
    struct Part {
        const char *name;
        int32_t *out;
        size_t bytes;
    } parts[2] = {{"sort_kth_rank_l.index", sort_kth_rank_out, 4 * (size_t) n_sample_item},
                  {"accu_n_user_rank_l.index", accu_out, 4 * (size_t) n_sample_item * (size_t) (n_item + 1)}};
    for (const Part &pt : parts) {
        if (!pt.out) continue;
        const std::string p = fmt("%s/%s", dir, pt.name);
        Mapped m;
        if (int st = m.open(p.c_str())) return st;
        if (m.n != pt.bytes) {
            set_error("%s: %zu bytes, expected %zu", p.c_str(), m.n, pt.bytes);
            return RKR_ERR_IO;
        }
        std::memcpy(pt.out, m.p, m.n);
    }
    return RKR_OK;
}

int rkr_index_load_files(rkr_index *index, int32_t method, const char *index_dir, const char *dataset_name,
                         int32_t n_sample, int32_t n_sample_query, int32_t sample_topk) {
    if (!index || !index_dir || !dataset_name || n_sample <= 0) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    if (method != RKR_METHOD_QS && method != RKR_METHOD_QSRP_NORMAL_LP && method != RKR_METHOD_US) {
        set_error("unknown method %d", method);
        return RKR_ERR_INVALID;
    }
    // SampleSearch: QS and QSRPNormalLP read the "QS" index of the query-distribution ranks
    // (SampleSearchIndexName, NameTranslation.hpp:36-60; QS.hpp:274-277, QSRPNormalLP.hpp:303-306),
    // US the uniform-rank "US" index (US.hpp:229-232)
    const std::string ss = method == RKR_METHOD_US
                               ? fmt("%s/memory_index/US-%s-n_sample_%d.index", index_dir, dataset_name, n_sample)
                               : fmt("%s/memory_index/QS-%s-n_sample_%d-n_sample_query_%d-sample_topk_%d.index",
                                     index_dir, dataset_name, n_sample, n_sample_query, sample_topk);
    int64_t n_user = 0;
    if (int st = rkr_index_shape(index, &n_user, nullptr, nullptr)) return st;
    {
        Mapped m;
        SampleSearchView v;
        int st = m.open(ss.c_str());
        if (st == RKR_OK) st = v.parse(m, ss.c_str());
        if (st != RKR_OK) return st;
        if (v.n_sample != n_sample || v.n_user != n_user || !v.thr) {
            set_error("%s: n_sample %lld, n_user %lld%s; the index has %lld users and asks for %d samples", ss.c_str(),
                      (long long) v.n_sample, (long long) v.n_user, v.thr ? "" : ", no thresholds",
                      (long long) n_user, n_sample);
            return RKR_ERR_IO;
        }
        if (int st2 = rkr_index_load_sample_search(index, v.rank, n_sample, v.thr)) return st2;
    }
    if (method == RKR_METHOD_US) return RKR_OK;
    const std::string svd = fmt("%s/svd_index/%s.index", index_dir, dataset_name);
    {
        Mapped m;
        SvdView v;
        int st = m.open(svd.c_str());
        if (st == RKR_OK) st = v.parse(m, svd.c_str());
        if (st != RKR_OK) return st;
        if (v.n_user != n_user) {
            set_error("%s: %lld users, the index has %lld", svd.c_str(), (long long) v.n_user, (long long) n_user);
            return RKR_ERR_IO;
        }
        if (method == RKR_METHOD_QS) return rkr_index_set_check_dim(index, v.check_dim);
        if (int st2 = rkr_index_load_svd(index, v.check_dim, v.transfer, v.user)) return st2;
    }
    // RegressionIndexName("QSRPNormalLP") is "QS" (NameTranslation.hpp; QSRPNormalLP.hpp:309-312)
    const std::string reg =
        fmt("%s/memory_index/NormalLinearRegressionLP-QS-%s-n_sample_%d-n_sample_query_%d-sample_topk_%d.index",
            index_dir, dataset_name, n_sample, n_sample_query, sample_topk);
    Mapped m;
    RegressionView v;
    int st = m.open(reg.c_str());
    if (st == RKR_OK) st = v.parse(m, reg.c_str());
    if (st != RKR_OK) return st;
    if (v.n_user != n_user || v.n_sample != n_sample) {
        set_error("%s: n_sample %d, n_user %lld; expected %d and %lld", reg.c_str(), v.n_sample, (long long) v.n_user,
                  n_sample, (long long) n_user);
        return RKR_ERR_IO;
    }
    std::vector<float> rec((size_t) 7 * (size_t) n_user);
    v.records(rec.data());
    return rkr_index_load_regression(index, v.rank, v.n_sample, rec.data());
}

// BuildScoreTableBatch (src/app/BuildScoreTableBatch.cpp:75-150) with ReadAll's writer
// (src/include/alg/DiskIndex/ReadAll.hpp: BuildIndexLoop): the first n_user_out users' score rows,
// each sorted descending, n_item floats per row in user order, no header.  The rows come from the
// device (rkr_score_sort_batch) a batch of at most 256 MB at a time.
int rkr_file_write_score_table(rkr_index *index, const char *path, int64_t n_user_out) {
    int64_t n_user = 0, n_item = 0;
    if (!index || !path || rkr_index_shape(index, &n_user, &n_item, nullptr) != RKR_OK || n_user_out < 0 ||
        n_user_out > n_user || n_item <= 0) {
        set_error("invalid argument");
        return RKR_ERR_INVALID;
    }
    Writer w;
    if (int st = w.open(path)) return st;
    const int64_t batch = std::max<int64_t>(1, (int64_t(256) << 20) / (n_item * (int64_t) sizeof(float)));
    std::vector<float> rows;
    for (int64_t u0 = 0; u0 < n_user_out; u0 += batch) {
        const int64_t nb = std::min(batch, n_user_out - u0);
        rows.resize((size_t) (nb * n_item));
        if (int st = rkr_score_sort_batch(index, u0, nb, rows.data())) return st;
        w.put(rows.data(), rows.size() * sizeof(float));
    }
    return w.close();
}

}  // extern "C"
