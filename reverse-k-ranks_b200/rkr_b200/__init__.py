"""Python binding of librkr_b200.so, the B200 reverse k-ranks engine (C ABI: include/rkr.h).

Mirrors the reference's index / query interface (DBGroup-SUSTech/reverse-k-ranks):

* ``Index`` is the device-resident index behind ``BaseIndex``
  (src/include/struct/MethodBase.hpp:14-27): it owns the users and items, the SampleSearch
  thresholds, the NormalLinearRegressionLP models and the SVD transform, and answers
  ``retrieval(method, query, topk)`` for the reference's ``QS``, ``QSRPNormalLP`` and ``US`` methods.
* The module-level functions are the reference's host-side index-build steps
  (normalisation, sampled items, k-th ranks, sample-rank selection, regression fit, SVD).

Errors raise ``RkrError`` with the library's message (the reference exits the process instead).
There is no CPU fallback: without the compiled library the import fails.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RKR_B200_LIB", os.path.join(os.path.dirname(_HERE), "librkr_b200.so"))

USER_RANK = np.dtype([("user_id", np.int32), ("rank", np.int32), ("query_ip", np.float32)])
QUERY_STATS = np.dtype([("n_prune", np.int32), ("n_result", np.int32), ("n_refine", np.int32),
                        ("n_candidate", np.int32), ("n_compute_item", np.int64), ("ip_cost", np.int64)])

METHODS = {"QS": 0, "QSRPNormalLP": 1, "US": 2}

RKR_OK, RKR_ERR_INVALID, RKR_ERR_CUDA, RKR_ERR_NOMEM, RKR_ERR_STATE, RKR_ERR_IO = 0, -1, -2, -3, -4, -5

# Every entry point declared in include/rkr.h.
EXPORTS = [
    "rkr_last_error", "rkr_version", "rkr_index_create", "rkr_index_destroy", "rkr_index_set_check_dim",
    "rkr_index_load_sample_search", "rkr_index_load_regression", "rkr_index_load_svd", "rkr_index_reset_state",
    "rkr_index_size_bytes", "rkr_index_build_sample_search", "rkr_retrieval", "rkr_retrieval_device",
    "rkr_score_sort_batch", "rkr_index_query_rank_distribution", "rkr_normalize", "rkr_sample_item",
    "rkr_sort_kth_rank", "rkr_find_optimal_sample_rank", "rkr_uniform_sample_rank", "rkr_fit_regression",
    "rkr_svd_build", "rkr_profile_enable", "rkr_profile_read", "rkr_build_thresholds_static",
    "rkr_index_level_tables", "rkr_query", "rkr_query_device", "rkr_server_create", "rkr_server_submit",
    "rkr_server_wait", "rkr_server_counters", "rkr_server_destroy", "rkr_score_estimates", "rkr_index_shape",
    "rkr_file_sample_search_info", "rkr_file_read_sample_search", "rkr_file_write_sample_search",
    "rkr_file_regression_info", "rkr_file_read_regression", "rkr_file_write_regression", "rkr_file_svd_info",
    "rkr_file_read_svd", "rkr_file_write_svd", "rkr_file_write_query_distribution",
    "rkr_file_read_query_distribution", "rkr_index_load_files", "rkr_index_set_shard", "rkr_shard_query",
    "rkr_shard_merge", "rkr_host_exchange_create", "rkr_host_exchange", "rkr_host_exchange_destroy",
    "rkr_index_fit_regression", "rkr_index_svd_build", "rkr_file_write_score_table", "rkr_index_insert_users",
    "rkr_index_delete_users", "rkr_index_svd_read",
]

# rkr_exchange_fn (include/rkr.h): int (*)(void *ctx, int32_t *counts, int64_t n, void *stream)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)


class RkrError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"rkr status {status}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"librkr_b200.so not found at {LIB_PATH}; build it with `make -C reverse-k-ranks_b200` "
                          "(or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    lib.rkr_last_error.restype = C.c_char_p
    lib.rkr_version.restype = C.c_int
    return lib


_lib = _load()


def lib():
    return _lib


def _check(status):
    if status != RKR_OK:
        raise RkrError(status, _lib.rkr_last_error().decode(errors="replace"))


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ---- host-side build steps ------------------------------------------------------------------------------

def normalize(v):
    """VectorMatrix::vectorNormalize (src/include/struct/VectorMatrix.hpp:51-66) on a copy."""
    v = _f32(v).copy()
    _check(_lib.rkr_normalize(_p(v), C.c_int64(v.shape[0]), C.c_int32(v.shape[1])))
    return v


def sample_item(n_item, n_sample_item):
    """SampleItem (src/app/build-index/QueryRankBySample.hpp:20-37)."""
    out = np.empty(n_sample_item, np.int32)
    _check(_lib.rkr_sample_item(C.c_int32(n_item), C.c_int32(n_sample_item), _p(out)))
    return out


def sort_kth_rank(accu, sample_topk):
    """ComputeSortKthRank (QueryRankBySample.hpp:103-134): (sorted k-th ranks, sample order)."""
    accu = _i32(accu)
    kth = np.empty(accu.shape[0], np.int32)
    sid = np.empty(accu.shape[0], np.int32)
    _check(_lib.rkr_sort_kth_rank(_p(accu), C.c_int64(accu.shape[1] - 1), C.c_int32(accu.shape[0]),
                                  C.c_int32(sample_topk), _p(kth), _p(sid)))
    return kth, sid


def find_optimal_sample_rank(n_user, n_item, n_sample, sort_kth, accu_sorted):
    """FindOptimalSampleFast, OptimalPart (OptimalSampleRankFast.hpp:269-472): (ranks, train cost)."""
    sk, acc = _i32(sort_kth), _i32(accu_sorted)
    out = np.empty(n_sample, np.int32)
    cost = np.zeros(1, np.int64)
    _check(_lib.rkr_find_optimal_sample_rank(C.c_int64(n_user), C.c_int64(n_item), C.c_int32(n_sample),
                                             C.c_int32(sk.shape[0]), _p(sk), _p(acc), _p(out), _p(cost)))
    return out, int(cost[0])


def uniform_sample_rank(n_item, n_sample):
    """FindUniformSample (UniformSample.hpp:17-56)."""
    out = np.empty(n_sample, np.int32)
    _check(_lib.rkr_uniform_sample_rank(C.c_int32(n_item), C.c_int32(n_sample), _p(out)))
    return out


def fit_regression(thresholds):
    """NormalLinearRegressionLP fit: [n_user][7] records (a, b, mu, sigma, error, smax, smin)."""
    thr = _f32(thresholds)
    out = np.empty((thr.shape[0], 7), np.float32)
    _check(_lib.rkr_fit_regression(_p(thr), C.c_int64(thr.shape[0]), C.c_int32(thr.shape[1]), _p(out)))
    return out


def svd_build(user, sigma=0.7):
    """SVD::PerformSVD (src/include/alg/SVD.hpp:62-124): (transfer_item, svd_user, check_dim)."""
    user = _f32(user)
    d = user.shape[1]
    ti = np.empty((d, d), np.float32)
    su = np.empty_like(user)
    cd = np.zeros(1, np.int32)
    _check(_lib.rkr_svd_build(_p(user), C.c_int64(user.shape[0]), C.c_int32(d), C.c_float(sigma), _p(ti), _p(su),
                              _p(cd)))
    return ti, su, int(cd[0])


def build_thresholds_static(d_user, n_user, d_item, n_item, dim, sample_rank, d_thresholds, stream=None):
    """rkr_build_thresholds_static: thresholds for users/items already on the current device
    (device pointers as ints), without any device allocation by the library; see include/rkr.h."""
    sr = _i32(sample_rank)
    _check(_lib.rkr_build_thresholds_static(C.c_void_p(d_user), C.c_int64(n_user), C.c_void_p(d_item),
                                            C.c_int64(n_item), C.c_int32(dim), _p(sr), C.c_int32(sr.shape[0]),
                                            C.c_void_p(d_thresholds), C.c_void_p(stream or 0)))


# ---- index files (the reference's on-disk layouts) ------------------------------------------------------

def _b(path):
    return os.fsencode(path)


def read_sample_search(path):
    """SampleSearch::LoadIndex file -> (ranks, thresholds [n_user][n_sample] or None, n_item)."""
    s, ni, nu, has = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int32()
    _check(_lib.rkr_file_sample_search_info(_b(path), C.byref(s), C.byref(ni), C.byref(nu), C.byref(has)))
    rank = np.empty(s.value, np.int32)
    thr = np.empty((nu.value, s.value), np.float32) if has.value else None
    _check(_lib.rkr_file_read_sample_search(_b(path), _p(rank), _p(thr)))
    return rank, thr, ni.value


def write_sample_search(path, sample_rank, n_item, thresholds=None, n_user=None):
    """SampleSearch::SaveIndex layout; thresholds None writes the ranks-only (qrs_to_sample_index) form."""
    sr = _i32(sample_rank)
    thr = None if thresholds is None else _f32(thresholds)
    nu = thr.shape[0] if thr is not None else int(n_user or 0)
    _check(_lib.rkr_file_write_sample_search(_b(path), _p(sr), C.c_int32(sr.shape[0]), C.c_int64(n_item),
                                             C.c_int64(nu), _p(thr)))


def read_regression(path):
    """NormalLinearRegressionLP::LoadIndex file -> (ranks, records [n_user][7], n_item)."""
    s, ni, nu = C.c_int32(), C.c_int64(), C.c_int64()
    _check(_lib.rkr_file_regression_info(_b(path), C.byref(s), C.byref(ni), C.byref(nu)))
    rank = np.empty(s.value, np.int32)
    rec = np.empty((nu.value, 7), np.float32)
    _check(_lib.rkr_file_read_regression(_b(path), _p(rank), _p(rec)))
    return rank, rec, ni.value


def write_regression(path, sample_rank, records, n_item):
    sr, rec = _i32(sample_rank), _f32(records)
    _check(_lib.rkr_file_write_regression(_b(path), _p(sr), C.c_int32(sr.shape[0]), C.c_int64(n_item),
                                          C.c_int64(rec.shape[0]), _p(rec)))


def read_svd(path, with_items=False):
    """SVD::LoadIndex file -> dict(transfer_item, svd_user, svd_item or None, check_dim, sigma, n_item)."""
    nu, ni, d, sg, cd = C.c_int64(), C.c_int64(), C.c_int32(), C.c_float(), C.c_int32()
    _check(_lib.rkr_file_svd_info(_b(path), C.byref(nu), C.byref(ni), C.byref(d), C.byref(sg), C.byref(cd)))
    ti = np.empty((d.value, d.value), np.float32)
    su = np.empty((nu.value, d.value), np.float32)
    si = np.empty((ni.value, d.value), np.float32) if with_items else None
    _check(_lib.rkr_file_read_svd(_b(path), _p(ti), _p(su), _p(si)))
    return dict(transfer_item=ti, svd_user=su, svd_item=si, check_dim=cd.value, sigma=sg.value, n_item=ni.value)


def write_svd(path, transfer_item, svd_user, check_dim, n_item, sigma=0.7, svd_item=None):
    ti, su = _f32(transfer_item), _f32(svd_user)
    si = None if svd_item is None else _f32(svd_item)
    _check(_lib.rkr_file_write_svd(_b(path), C.c_int64(su.shape[0]), C.c_int64(n_item), C.c_int32(su.shape[1]),
                                   C.c_float(sigma), C.c_int32(check_dim), _p(ti), _p(su), _p(si)))


def write_query_distribution(dirname, sample_item, sort_kth_rank, sort_sample_id, accu):
    """WriteDistributionBelowTopk's directory from the build steps' outputs (accu in sample order)."""
    si, sk, sid, acc = _i32(sample_item), _i32(sort_kth_rank), _i32(sort_sample_id), _i32(accu)
    _check(_lib.rkr_file_write_query_distribution(_b(dirname), _p(si), _p(sk), _p(sid), _p(acc),
                                                  C.c_int32(si.shape[0]), C.c_int64(acc.shape[1] - 1)))


def read_query_distribution(dirname, n_sample_item, n_item):
    """-> (sampled item ids, sorted k-th ranks, accu rows), all in the files' (sorted-sample) order."""
    si = np.empty(n_sample_item, np.int32)
    sk = np.empty(n_sample_item, np.int32)
    acc = np.empty((n_sample_item, n_item + 1), np.int32)
    _check(_lib.rkr_file_read_query_distribution(_b(dirname), C.c_int32(n_sample_item), C.c_int64(n_item), _p(si),
                                                 _p(sk), _p(acc)))
    return si, sk, acc


# ---- the device index ---------------------------------------------------------------------------------------

class Index:
    """Device-resident reverse k-ranks index (QS / QSRPNormalLP / US)."""

    def __init__(self, user, item, device: int = 0):
        user, item = _f32(user), _f32(item)
        if user.ndim != 2 or item.ndim != 2 or user.shape[1] != item.shape[1]:
            raise ValueError("user and item must be 2-D with the same dimension")
        self.n_user, self.dim = user.shape
        self.n_item = item.shape[0]
        h = C.c_void_p()
        _check(_lib.rkr_index_create(C.c_int32(device), _p(user), C.c_int64(self.n_user), _p(item),
                                     C.c_int64(self.n_item), C.c_int32(self.dim), C.byref(h)))
        self._h = h
        self.n_sample = 0

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.rkr_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_check_dim(self, check_dim):
        _check(_lib.rkr_index_set_check_dim(self._h, C.c_int32(check_dim)))

    def load_sample_search(self, sample_rank, thresholds):
        sr, thr = _i32(sample_rank), _f32(thresholds)
        _check(_lib.rkr_index_load_sample_search(self._h, _p(sr), C.c_int32(sr.shape[0]), _p(thr)))
        self.n_sample = sr.shape[0]

    def build_sample_search(self, sample_rank, return_thresholds=True):
        sr = _i32(sample_rank)
        out = np.empty((self.n_user, sr.shape[0]), np.float32) if return_thresholds else None
        _check(_lib.rkr_index_build_sample_search(self._h, _p(sr), C.c_int32(sr.shape[0]), _p(out)))
        self.n_sample = sr.shape[0]
        return out

    def load_regression(self, sample_rank, records):
        sr, rec = _i32(sample_rank), _f32(records)
        _check(_lib.rkr_index_load_regression(self._h, _p(sr), C.c_int32(sr.shape[0]), _p(rec)))

    def fit_regression(self, records=True):
        """rkr_index_fit_regression: fit the regression models on the device from the resident
        thresholds and make them the index's; returns the [n_user][7] records (or None)."""
        out = np.empty((self.n_user, 7), np.float32) if records else None
        _check(_lib.rkr_index_fit_regression(self._h, _p(out)))
        return out

    def svd_build(self, sigma=0.7, copy_out=True):
        """rkr_index_svd_build: the SVD transform from the resident users on the device, made the
        index's; returns (transfer_item, svd_user, check_dim) (the arrays None without copy_out)."""
        ti = np.empty((self.dim, self.dim), np.float32) if copy_out else None
        su = np.empty((self.n_user, self.dim), np.float32) if copy_out else None
        cd = C.c_int32()
        _check(_lib.rkr_index_svd_build(self._h, C.c_float(sigma), _p(ti), _p(su), C.byref(cd)))
        return ti, su, cd.value

    def load_svd(self, check_dim, transfer_item, svd_user):
        ti, su = _f32(transfer_item), _f32(svd_user)
        _check(_lib.rkr_index_load_svd(self._h, C.c_int32(check_dim), _p(ti), _p(su)))

    def reset_state(self):
        _check(_lib.rkr_index_reset_state(self._h))

    def load_files(self, method, index_dir, dataset_name, n_sample, n_sample_query=0, sample_topk=0):
        """The file set the reference's factories read (rkr_index_load_files)."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        _check(_lib.rkr_index_load_files(self._h, C.c_int32(m), _b(index_dir), _b(dataset_name), C.c_int32(n_sample),
                                         C.c_int32(n_sample_query), C.c_int32(sample_topk)))
        self.n_sample = n_sample

    def score_estimates(self, method, query):
        """The tensor-core pair scores' estimates and bounds (rkr_score_estimates): [n_query][n_user][2]."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        q = _f32(query)
        out = np.empty((q.shape[0], self.n_user, 2), np.float32)
        _check(_lib.rkr_score_estimates(self._h, C.c_int32(m), _p(q), C.c_int32(q.shape[0]), _p(out)))
        return out

    def level_tables(self):
        """The regression models' level-boundary tables (rkr_index_level_tables): (levels L_g [16], array
        [n_user][2][16][2] of (boundary score, guard band))."""
        lv = np.zeros(16, np.int32)
        out = np.empty((self.n_user, 2, 16, 2), np.float32)
        _check(_lib.rkr_index_level_tables(self._h, _p(lv), _p(out)))
        return lv, out

    def size_bytes(self):
        v = C.c_uint64()
        _check(_lib.rkr_index_size_bytes(self._h, C.byref(v)))
        return v.value

    def retrieval(self, method, query, topk, stats=False, out=None):
        """BaseIndex::Retrieval: [n_answered][topk] USER_RANK records (and QUERY_STATS per query).

        `out`, if given, is the caller's C-contiguous USER_RANK array of at least n_query x topk
        records (for instance one buffer in pinned host memory reused across calls); the result is a
        view of it."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        q = _f32(query)
        nq = q.shape[0]
        n_rows = max(nq, 100)
        if out is None:
            out = np.zeros((n_rows, topk), USER_RANK)
        else:
            if out.dtype != USER_RANK or not out.flags.c_contiguous or out.size < nq * topk:
                raise ValueError(f"out must be a C-contiguous USER_RANK array of at least {nq} x {topk} records")
            out = out.reshape(-1)[: nq * topk].reshape(nq, topk)
        st = np.zeros(n_rows, QUERY_STATS) if stats else None
        na = C.c_int32()
        _check(_lib.rkr_retrieval(self._h, C.c_int32(m), _p(q), C.c_int32(nq), C.c_int32(topk), _p(out), _p(st),
                                  C.byref(na)))
        n = na.value
        return (out[:n], st[:n]) if stats else out[:n]

    def query(self, method, query, k_per_q, stats=False):
        """Retrieval with a top-k per query (rkr_query): a list of [k_i] USER_RANK arrays, one per
        answered query (and the QUERY_STATS per query)."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        q = _f32(query)
        ks = _i32(k_per_q)
        if ks.shape[0] != q.shape[0]:
            raise ValueError("one k per query")
        out = np.zeros(int(ks.sum()), USER_RANK)
        st = np.zeros(max(q.shape[0], 1), QUERY_STATS) if stats else None
        na = C.c_int32()
        _check(_lib.rkr_query(self._h, C.c_int32(m), _p(q), C.c_int32(q.shape[0]), _p(ks), _p(out), _p(st),
                              C.byref(na)))
        n = na.value
        off = np.concatenate([[0], np.cumsum(ks[:n])])
        rows = [out[off[i]:off[i + 1]] for i in range(n)]
        return (rows, st[:n]) if stats else rows

    def query_device(self, method, d_query, n_query, k_per_q, d_out, d_stats=None, stream=None):
        """Same with device pointers (ints) for queries and outputs; k_per_q a host array."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        ks = _i32(k_per_q)
        na = C.c_int32()
        _check(_lib.rkr_query_device(self._h, C.c_int32(m), C.c_void_p(d_query), C.c_int32(n_query), _p(ks),
                                     C.c_void_p(d_out), C.c_void_p(d_stats or 0), C.byref(na),
                                     C.c_void_p(stream or 0)))
        return na.value

    def retrieval_device(self, method, d_query, n_query, topk, d_out, d_stats=None, stream=None):
        """Same with device pointers (ints): queries [n_query][dim] f32, out [n][topk] USER_RANK."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        na = C.c_int32()
        _check(_lib.rkr_retrieval_device(self._h, C.c_int32(m), C.c_void_p(d_query), C.c_int32(n_query),
                                         C.c_int32(topk), C.c_void_p(d_out), C.c_void_p(d_stats or 0),
                                         C.byref(na), C.c_void_p(stream or 0)))
        return na.value

    def profile(self, on=True):
        """Turn per-kernel event timing on or off (rkr_profile_enable)."""
        _check(_lib.rkr_profile_enable(self._h, C.c_int32(1 if on else 0)))

    def profile_read(self):
        """{kernel name: (total ms, launches)} since the previous read."""
        n = C.c_int32()
        _check(_lib.rkr_profile_read(self._h, C.c_int32(0), None, None, None, C.byref(n)))
        k = n.value
        names = C.create_string_buffer(64 * max(k, 1))
        ms = np.zeros(max(k, 1), np.float64)
        cnt = np.zeros(max(k, 1), np.int64)
        _check(_lib.rkr_profile_read(self._h, C.c_int32(k), names, _p(ms), _p(cnt), C.byref(n)))
        return {names.raw[64 * i:64 * i + 64].split(b"\0")[0].decode(): (float(ms[i]), int(cnt[i])) for i in range(k)}

    def svd_read(self):
        """rkr_index_svd_read: (transfer_item, svd_user, check_dim) of the index's SVD transform."""
        ti = np.empty((self.dim, self.dim), np.float32)
        su = np.empty((self.n_user, self.dim), np.float32)
        cd = C.c_int32()
        _check(_lib.rkr_index_svd_read(self._h, _p(ti), _p(su), C.byref(cd)))
        return ti, su, cd.value

    def insert_users(self, user, sigma=0.7):
        """rkr_index_insert_users: append normalised users (thresholds, models, SVD rebuilt on the device)."""
        u = _f32(user)
        if u.ndim != 2 or u.shape[1] != self.dim:
            raise ValueError("users must be [n][dim]")
        _check(_lib.rkr_index_insert_users(self._h, _p(u), C.c_int64(u.shape[0]), C.c_float(sigma)))
        self.n_user += u.shape[0]

    def delete_users(self, ids):
        """rkr_index_delete_users: remove users by id (the rest close up in order)."""
        d = np.ascontiguousarray(ids, dtype=np.int64)
        _check(_lib.rkr_index_delete_users(self._h, _p(d), C.c_int64(d.shape[0])))
        self.n_user -= d.shape[0]

    def write_score_table(self, path, n_user_out=None):
        """rkr_file_write_score_table: bstb's disk score table (descending rows, no header)."""
        n = self.n_user if n_user_out is None else int(n_user_out)
        _check(_lib.rkr_file_write_score_table(self._h, _b(path), C.c_int64(n)))

    def score_sort_batch(self, start_user, n_rows):
        """ComputeScoreTableBatch::ComputeSortItemsBatch: descending score rows of users [start, start+n)."""
        out = np.empty((n_rows, self.n_item), np.float32)
        _check(_lib.rkr_score_sort_batch(self._h, C.c_int64(start_user), C.c_int64(n_rows), _p(out)))
        return out

    def query_rank_distribution(self, sample_item_ids):
        """ComputeQueryRankByComputation: accumulated user counts by rank, [n_sample_item][n_item+1]
        (on a user shard: every shard's users, each shard calling)."""
        si = _i32(sample_item_ids)
        out = np.empty((si.shape[0], self.n_item + 1), np.int32)
        _check(_lib.rkr_index_query_rank_distribution(self._h, _p(si), C.c_int32(si.shape[0]), _p(out)))
        return out

    # ---- user shards ----

    def set_shard(self, shard, n_shards, user_offset, n_user_total, exchange):
        """rkr_index_set_shard: this index becomes shard `shard` of n_shards, holding users
        [user_offset, user_offset + n_user) of n_user_total.  exchange: a HostExchange, an
        (EXCHANGE_FN, ctx) pair, or a Python callable fn(counts_address, n, stream) that sums the n
        int32 counts over all shards in place (see rkr_b200.shard.TorchExchange); None with
        n_shards == 1 makes the index whole again."""
        if exchange is None:
            fn, ctx, keep = None, None, None
        elif isinstance(exchange, HostExchange):
            fn, ctx, keep = exchange.fn, exchange.ctx, exchange
        elif isinstance(exchange, tuple):
            fn, ctx = exchange
            keep = exchange
        else:
            fn, ctx = exchange_callback(exchange), None
            keep = (fn, exchange)
        _check(_lib.rkr_index_set_shard(self._h, C.c_int32(shard), C.c_int32(n_shards), C.c_int64(user_offset),
                                        C.c_int64(n_user_total), fn, C.c_void_p(ctx)))
        self._exchange_keep = keep  # the callback must outlive its use

    def shard_query(self, method, query, k_per_q, stats=False):
        """rkr_shard_query: this shard's part of rkr_query -- (part, n_front[, stats]) with part the
        flat sum(k) USER_RANK entries (row q: n_front[q] results, then candidates; user_id -1 unused)."""
        m = METHODS[method] if isinstance(method, str) else int(method)
        q = _f32(query)
        ks = _i32(k_per_q)
        if ks.shape[0] != q.shape[0]:
            raise ValueError("one k per query")
        part = np.zeros(int(ks.sum()), USER_RANK)
        front = np.zeros(max(q.shape[0], 1), np.int32)
        st = np.zeros(max(q.shape[0], 1), QUERY_STATS) if stats else None
        na = C.c_int32()
        _check(_lib.rkr_shard_query(self._h, C.c_int32(m), _p(q), C.c_int32(q.shape[0]), _p(ks), _p(part), _p(front),
                                    _p(st), C.byref(na)))
        n = na.value
        part = part[:int(ks[:n].sum())]
        return (part, front[:n], st[:n]) if stats else (part, front[:n])


# ---- user shards ------------------------------------------------------------------------------------------

def exchange_callback(fn):
    """An rkr_exchange_fn calling fn(counts_address, n, stream) (stream 0: host memory); an exception
    fails the query.  Keep the returned object alive while an index uses it."""
    def cb(ctx, counts, n, stream):
        try:
            fn(counts or 0, int(n), stream or 0)
            return 0
        except Exception:  # noqa: BLE001 -- reported to the library as a failed exchange
            return 1
    return EXCHANGE_FN(cb)


class HostExchange:
    """rkr_host_exchange: the count exchange of shards driven by threads of one process (for example
    several shards on one GPU).  Waits up to timeout_s for every member at each exchange."""

    def __init__(self, n_members, timeout_s=60.0):
        g = C.c_void_p()
        _check(_lib.rkr_host_exchange_create(C.c_int32(n_members), C.c_double(timeout_s), C.byref(g)))
        self._g = g
        self.fn = C.cast(_lib.rkr_host_exchange, EXCHANGE_FN)

    @property
    def ctx(self):
        return self._g.value

    def close(self):
        if getattr(self, "_g", None) is not None and self._g.value:
            _lib.rkr_host_exchange_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def shard_merge(k_per_q, parts, fronts, stats=None):
    """rkr_shard_merge: the shards' parts (in shard order) merged into rkr_query's output: a flat
    sum(k) USER_RANK array (and the merged QUERY_STATS when every shard's stats are given)."""
    ks = _i32(k_per_q)
    n_sh, nq = len(parts), ks.shape[0]
    parts = [np.ascontiguousarray(p, USER_RANK) for p in parts]
    fronts = [_i32(f) for f in fronts]
    for p, f in zip(parts, fronts):
        if p.shape[0] != int(ks.sum()) or f.shape[0] != nq:
            raise ValueError("every part holds sum(k_per_q) entries and every n_front one per query")
    pp = (C.c_void_p * n_sh)(*[p.ctypes.data for p in parts])
    fp = (C.c_void_p * n_sh)(*[f.ctypes.data for f in fronts])
    sp, st_out = None, None
    if stats is not None:
        stats = [np.ascontiguousarray(s, QUERY_STATS) for s in stats]
        sp = (C.c_void_p * n_sh)(*[s.ctypes.data for s in stats])
        st_out = np.zeros(max(nq, 1), QUERY_STATS)
    out = np.zeros(int(ks.sum()), USER_RANK)
    _check(_lib.rkr_shard_merge(C.c_int32(n_sh), C.c_int32(nq), _p(ks), pp, fp, sp, _p(out), _p(st_out)))
    return (out, st_out[:nq]) if stats is not None else out


# ---- serving ----------------------------------------------------------------------------------------------

class _ServerConfig(C.Structure):
    _fields_ = [("method", C.c_int32), ("max_batch_queries", C.c_int32), ("n_workers", C.c_int32),
                ("reserved", C.c_int32), ("workspace_bytes", C.c_int64)]


class Server:
    """A persistent serving loop over a resident Index (rkr_server_*): submit() queues a request of
    query items with a top-k per item and returns a ticket; wait(ticket) returns its rows as
    Index.query would for the request alone on a fresh index."""

    def __init__(self, index, method="QSRPNormalLP", max_batch_queries=1024, n_workers=2, workspace_bytes=0):
        self.index = index
        cfg = _ServerConfig(METHODS[method] if isinstance(method, str) else int(method), int(max_batch_queries),
                            int(n_workers), 0, int(workspace_bytes))
        h = C.c_void_p()
        _check(_lib.rkr_server_create(index.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self._k = {}

    def submit(self, query, k_per_q):
        q = _f32(query)
        ks = _i32(k_per_q)
        if q.ndim != 2 or ks.shape[0] != q.shape[0]:
            raise ValueError("query [n][dim] and one k per query item")
        t = C.c_uint64()
        _check(_lib.rkr_server_submit(self._h, _p(q), C.c_int32(q.shape[0]), _p(ks), C.byref(t)))
        self._k[t.value] = ks
        return t.value

    def wait(self, ticket, timeout=-1.0, stats=False):
        """(rows, latency {done, start} in seconds[, stats]): rows a list of [k_i] USER_RANK arrays."""
        ks = self._k.pop(ticket)
        out = np.zeros(int(ks.sum()), USER_RANK)
        st = np.zeros(ks.shape[0], QUERY_STATS)
        lat = np.zeros(2, np.float64)
        _check(_lib.rkr_server_wait(self._h, C.c_uint64(ticket), C.c_double(timeout), _p(out), _p(st), _p(lat)))
        off = np.concatenate([[0], np.cumsum(ks)])
        rows = [out[off[i]:off[i + 1]] for i in range(ks.shape[0])]
        lat = {"done": float(lat[0]), "start": float(lat[1])}
        return (rows, lat, st) if stats else (rows, lat)

    def counters(self):
        v = [C.c_int64() for _ in range(4)]
        busy = C.c_double()
        _check(_lib.rkr_server_counters(self._h, *[C.byref(x) for x in v], C.byref(busy)))
        return {"batches": v[0].value, "requests": v[1].value, "queries": v[2].value, "padded": v[3].value,
                "busy_s": busy.value}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.rkr_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
