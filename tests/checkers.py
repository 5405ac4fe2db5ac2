"""ctypes bindings of the two checkers used by the parity tests (test infrastructure).

* ``Oracle``    -- oracle/librkr_oracle.so, the C restatement of the reference path (rkr_oracle.c).
* ``Reference`` -- oracle/_ref/librkr_ref.so, the reference's own headers compiled by
  oracle/Makefile (present only where it was built from the reference sources).

Both take and return numpy arrays; nothing here touches a GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "librkr_oracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "librkr_ref.so")
REF_FAST_SO = os.path.join(ORACLE_DIR, "_ref", "librkr_ref_fast.so")  # -Ofast, timing only


def reference_root() -> str:
    """The reference checkout (read-only): $RKR_REFERENCE_ROOT, else a `reference` directory beside
    this repository.  Only the fixture generators and the CPU-side tests read it; nothing that runs
    on the GPU needs it."""
    return os.environ.get("RKR_REFERENCE_ROOT") or os.path.normpath(os.path.join(ROOT, "..", "reference"))


USER_RANK = np.dtype([("user_id", np.int32), ("rank", np.int32), ("query_ip", np.float32)])
STATS = np.dtype([("n_prune", np.int32), ("n_result", np.int32), ("n_refine", np.int32),
                  ("n_candidate", np.int32), ("n_compute_item", np.int64), ("ip_cost", np.int64)])


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def build_oracle() -> str:
    """Compile the C restatement (it is source in the repository) if its library is missing."""
    src = os.path.join(ORACLE_DIR, "rkr_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", ORACLE_DIR, "CC=gcc", "librkr_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return ORACLE_SO


class Oracle:
    def __init__(self):
        self.lib = C.CDLL(build_oracle())
        L = self.lib
        L.orc_cdf_phi.restype = C.c_float
        L.orc_cdf_phi.argtypes = [C.c_float]
        L.orc_sqrt_constexpr.restype = C.c_float
        L.orc_sqrt_constexpr.argtypes = [C.c_float]
        L.orc_inner_product.restype = C.c_float
        for name in ("orc_qs_retrieval", "orc_us_retrieval", "orc_qsrp_retrieval", "orc_optimal_sample_rank",
                     "orc_qs_retrieval_shard", "orc_us_retrieval_shard", "orc_qsrp_retrieval_shard"):
            getattr(L, name).restype = C.c_int

    def normalize(self, v):
        v = _f32(v).copy()
        self.lib.orc_normalize(_p(v), C.c_int64(v.shape[0]), C.c_int32(v.shape[1]))
        return v

    def inner_product(self, a, b):
        a, b = _f32(a), _f32(b)
        return self.lib.orc_inner_product(_p(a), _p(b), C.c_int32(a.shape[0]))

    def cdf_phi(self, x):
        return np.float32(self.lib.orc_cdf_phi(C.c_float(float(x))))

    def score_sort_rows(self, user, item, start, n_rows):
        user, item = _f32(user), _f32(item)
        out = np.empty((n_rows, item.shape[0]), np.float32)
        self.lib.orc_score_sort_rows(_p(user), C.c_int64(start), C.c_int64(n_rows), _p(item),
                                     C.c_int64(item.shape[0]), C.c_int32(item.shape[1]), _p(out))
        return out

    def build_thresholds(self, user, item, sample_rank):
        user, item, sr = _f32(user), _f32(item), _i32(sample_rank)
        out = np.empty((user.shape[0], sr.shape[0]), np.float32)
        self.lib.orc_build_thresholds(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                      C.c_int32(user.shape[1]), _p(sr), C.c_int32(sr.shape[0]), _p(out))
        return out

    def query_rank_distribution(self, user, item, sample_item):
        user, item, si = _f32(user), _f32(item), _i32(sample_item)
        n_user, n_item = user.shape[0], item.shape[0]
        ranks = np.empty((n_user, si.shape[0]), np.int32)
        accu = np.empty((si.shape[0], n_item + 1), np.int32)
        self.lib.orc_query_rank_distribution(_p(user), C.c_int64(n_user), _p(item), C.c_int64(n_item),
                                             C.c_int32(user.shape[1]), _p(si), C.c_int32(si.shape[0]),
                                             _p(ranks), _p(accu))
        return ranks, accu

    def kth_rank(self, accu, sample_topk):
        accu = _i32(accu)
        out = np.empty(accu.shape[0], np.int32)
        self.lib.orc_kth_rank(_p(accu), C.c_int64(accu.shape[1] - 1), C.c_int32(accu.shape[0]),
                              C.c_int32(sample_topk), _p(out))
        return out

    def uniform_sample_rank(self, n_item, n_sample):
        out = np.empty(n_sample, np.int32)
        self.lib.orc_uniform_sample_rank(C.c_int32(n_item), C.c_int32(n_sample), _p(out))
        return out

    def optimal_sample_rank(self, n_user, n_item, n_sample, sort_kth, accu_sorted):
        sk, acc = _i32(sort_kth), _i32(accu_sorted)
        out = np.empty(n_sample, np.int32)
        cost = np.zeros(1, np.int64)
        rc = self.lib.orc_optimal_sample_rank(C.c_int64(n_user), C.c_int64(n_item), C.c_int32(n_sample),
                                              C.c_int32(sk.shape[0]), _p(sk), _p(acc), _p(out), _p(cost))
        assert rc == 0
        return out, int(cost[0])

    def fit_regression(self, thr):
        thr = _f32(thr)
        out = np.empty((thr.shape[0], 7), np.float32)
        self.lib.orc_fit_regression(_p(thr), C.c_int64(thr.shape[0]), C.c_int32(thr.shape[1]), _p(out))
        return out

    def regression_rank_bound(self, reg, reg_rank, n_item, user_ids, qlb, qub):
        reg, rr = _f32(reg), _i32(reg_rank)
        lb = np.empty(len(user_ids), np.int32)
        ub = np.empty(len(user_ids), np.int32)
        for i, (u, a, b) in enumerate(zip(user_ids, qlb, qub)):
            rec = reg[u]
            l = C.c_int32(); h = C.c_int32()
            self.lib.orc_regression_rank_bound(C.c_float(float(a)), C.c_float(float(b)), _p(rec[0:2].copy()),
                                               _p(rec[2:4].copy()), C.c_float(float(rec[4])), _p(rec[5:7].copy()),
                                               _p(rr), C.c_int32(rr.shape[0]), C.c_int64(n_item),
                                               C.byref(l), C.byref(h))
            lb[i], ub[i] = l.value, h.value
        return lb, ub

    def level_boundaries_at(self, rec, sample_rank, n_item, levels, side):
        """orc_level_boundaries_at: the smallest score whose rank-bound level is <= levels[g]."""
        rec, sr, lv = _f32(rec), _i32(sample_rank), _i32(levels)
        out = np.empty(lv.shape[0], np.float32)
        self.lib.orc_level_boundaries_at(_p(rec), _p(sr), C.c_int32(sr.shape[0]), C.c_int64(n_item), _p(lv),
                                         C.c_int32(side), C.c_int32(lv.shape[0]), _p(out))
        return out

    def level_boundaries(self, rec, sample_rank, n_item, stride, side, n_out):
        """orc_level_boundaries: the smallest score whose rank-bound level is <= g * stride."""
        rec, sr = _f32(rec), _i32(sample_rank)
        out = np.empty(n_out, np.float32)
        self.lib.orc_level_boundaries(_p(rec), _p(sr), C.c_int32(sr.shape[0]), C.c_int64(n_item), C.c_int32(stride),
                                      C.c_int32(side), C.c_int32(n_out), _p(out))
        return out

    def qs_retrieval(self, user, item, check_dim, sample_rank, thr, query, topk):
        user, item, sr, thr, query = _f32(user), _f32(item), _i32(sample_rank), _f32(thr), _f32(query)
        nq = query.shape[0]
        out = np.zeros((nq, topk), USER_RANK)
        st = np.zeros(nq, STATS)
        rc = self.lib.orc_qs_retrieval(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                       C.c_int32(user.shape[1]), C.c_int32(check_dim), _p(sr),
                                       C.c_int32(sr.shape[0]), _p(thr), _p(query), C.c_int32(nq),
                                       C.c_int32(topk), _p(out), _p(st))
        assert rc == 0
        return out, st

    def us_retrieval(self, user, item, sample_rank, thr, query, topk):
        user, item, sr, thr, query = _f32(user), _f32(item), _i32(sample_rank), _f32(thr), _f32(query)
        nq = query.shape[0]
        out = np.zeros((nq, topk), USER_RANK)
        st = np.zeros(nq, STATS)
        n = self.lib.orc_us_retrieval(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                      C.c_int32(user.shape[1]), _p(sr), C.c_int32(sr.shape[0]), _p(thr),
                                      _p(query), C.c_int32(nq), C.c_int32(topk), _p(out), _p(st))
        assert n >= 0
        return out[:n], st[:n]

    def qsrp_retrieval(self, user, svd_user, transfer_item, item, check_dim, sample_rank, thr, reg_rank, reg,
                       query, topk, qip_state=None):
        user, svd_user, ti, item = _f32(user), _f32(svd_user), _f32(transfer_item), _f32(item)
        sr, thr, rr, reg, query = _i32(sample_rank), _f32(thr), _i32(reg_rank), _f32(reg), _f32(query)
        nq, n_user = query.shape[0], user.shape[0]
        if qip_state is None:
            qip_state = np.zeros(n_user, np.float32)
        out = np.zeros((nq, topk), USER_RANK)
        st = np.zeros(nq, STATS)
        rc = self.lib.orc_qsrp_retrieval(_p(user), _p(svd_user), _p(ti), C.c_int64(n_user), _p(item),
                                         C.c_int64(item.shape[0]), C.c_int32(user.shape[1]),
                                         C.c_int32(check_dim), _p(sr), C.c_int32(sr.shape[0]), _p(thr),
                                         _p(rr), C.c_int32(rr.shape[0]), _p(reg), _p(query), C.c_int32(nq),
                                         C.c_int32(topk), _p(qip_state), _p(out), _p(st))
        assert rc == 0
        return out, st

    # ---- the same on one user shard (exchange: an (rkr_exchange_fn, ctx) pair summing host counts) ----

    def _shard_out(self, nq, topk):
        return np.zeros((nq, topk), USER_RANK), np.zeros(nq, np.int32), np.zeros(nq, STATS)

    def qs_retrieval_shard(self, user, item, check_dim, sample_rank, thr, query, topk, user_offset, n_user_total,
                           exchange):
        user, item, sr, thr, query = _f32(user), _f32(item), _i32(sample_rank), _f32(thr), _f32(query)
        nq = query.shape[0]
        out, front, st = self._shard_out(nq, topk)
        fn, ctx = exchange
        rc = self.lib.orc_qs_retrieval_shard(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                             C.c_int32(user.shape[1]), C.c_int32(check_dim), _p(sr),
                                             C.c_int32(sr.shape[0]), _p(thr), _p(query), C.c_int32(nq),
                                             C.c_int32(topk), C.c_int64(user_offset), C.c_int64(n_user_total),
                                             C.c_int32(user_offset == 0), fn, C.c_void_p(ctx), _p(out), _p(front),
                                             _p(st))
        assert rc == nq, rc
        return out, front, st

    def us_retrieval_shard(self, user, item, sample_rank, thr, query, topk, user_offset, n_user_total, exchange):
        user, item, sr, thr, query = _f32(user), _f32(item), _i32(sample_rank), _f32(thr), _f32(query)
        nq = query.shape[0]
        out, front, st = self._shard_out(nq, topk)
        fn, ctx = exchange
        n = self.lib.orc_us_retrieval_shard(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                            C.c_int32(user.shape[1]), _p(sr), C.c_int32(sr.shape[0]), _p(thr),
                                            _p(query), C.c_int32(nq), C.c_int32(topk), C.c_int64(user_offset),
                                            C.c_int64(n_user_total), C.c_int32(user_offset == 0), fn,
                                            C.c_void_p(ctx), _p(out), _p(front), _p(st))
        assert n >= 0, n
        return out[:n], front[:n], st[:n]

    def qsrp_retrieval_shard(self, user, svd_user, transfer_item, item, check_dim, sample_rank, thr, reg_rank, reg,
                             query, topk, user_offset, n_user_total, exchange, qip_state=None):
        user, svd_user, ti, item = _f32(user), _f32(svd_user), _f32(transfer_item), _f32(item)
        sr, thr, rr, reg, query = _i32(sample_rank), _f32(thr), _i32(reg_rank), _f32(reg), _f32(query)
        nq, n_user = query.shape[0], user.shape[0]
        if qip_state is None:
            qip_state = np.zeros(n_user, np.float32)
        out, front, st = self._shard_out(nq, topk)
        fn, ctx = exchange
        rc = self.lib.orc_qsrp_retrieval_shard(_p(user), _p(svd_user), _p(ti), C.c_int64(n_user), _p(item),
                                               C.c_int64(item.shape[0]), C.c_int32(user.shape[1]),
                                               C.c_int32(check_dim), _p(sr), C.c_int32(sr.shape[0]), _p(thr),
                                               _p(rr), C.c_int32(rr.shape[0]), _p(reg), _p(query), C.c_int32(nq),
                                               C.c_int32(topk), C.c_int64(user_offset), C.c_int64(n_user_total),
                                               C.c_int32(user_offset == 0), fn, C.c_void_p(ctx), _p(qip_state),
                                               _p(out), _p(front), _p(st))
        assert rc == nq, rc
        return out, front, st

    def exact_rank_f64(self, user, item, query):
        user, item, query = _f32(user), _f32(item), _f32(query)
        out = np.empty((query.shape[0], user.shape[0]), np.int32)
        self.lib.orc_exact_rank_f64(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                    C.c_int32(user.shape[1]), _p(query), C.c_int32(query.shape[0]), _p(out))
        return out


class Reference:
    """The reference's own code (oracle/_ref).  ``available()`` is False where it was not built."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self, n_thread: int = 1):
        self.lib = C.CDLL(REF_SO)
        self.lib.ref_inner_product.restype = C.c_float
        self.lib.ref_set_threads(C.c_int(n_thread))
        self.n_thread = n_thread

    def _tmp(self):
        return tempfile.TemporaryDirectory(prefix="rkr_ref_")

    def normalize(self, v):
        v = _f32(v).copy()
        self.lib.ref_normalize(_p(v), C.c_int64(v.shape[0]), C.c_int32(v.shape[1]))
        return v

    def build_thresholds(self, user, item, sample_rank):
        user, item, sr = _f32(user), _f32(item), _i32(sample_rank)
        out = np.empty((user.shape[0], sr.shape[0]), np.float32)
        self.lib.ref_build_thresholds(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                      C.c_int32(user.shape[1]), _p(sr), C.c_int32(sr.shape[0]), _p(out))
        return out

    def score_sort_rows(self, user, item, start, n_rows):
        user, item = _f32(user), _f32(item)
        out = np.empty((n_rows, item.shape[0]), np.float32)
        self.lib.ref_score_sort_rows(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                                     C.c_int32(user.shape[1]), C.c_int64(start), C.c_int64(n_rows), _p(out))
        return out

    def sample_item(self, n_item, n_sample_item):
        out = np.empty(n_sample_item, np.int32)
        self.lib.ref_sample_item(C.c_int32(n_item), C.c_int32(n_sample_item), _p(out))
        return out

    def query_rank_distribution(self, user, item, sample_item):
        user, item, si = _f32(user), _f32(item), _i32(sample_item)
        accu = np.empty((si.shape[0], item.shape[0] + 1), np.int32)
        self.lib.ref_query_rank_distribution(_p(user), C.c_int64(user.shape[0]), _p(item),
                                             C.c_int64(item.shape[0]), C.c_int32(user.shape[1]), _p(si),
                                             C.c_int32(si.shape[0]), _p(accu))
        return accu

    def sort_kth_rank(self, accu, sample_topk):
        accu = _i32(accu)
        kth = np.empty(accu.shape[0], np.int32)
        sid = np.empty(accu.shape[0], np.int32)
        self.lib.ref_sort_kth_rank(_p(accu), C.c_int64(accu.shape[1] - 1), C.c_int32(accu.shape[0]),
                                   C.c_int32(sample_topk), _p(kth), _p(sid))
        return kth, sid

    def find_optimal_sample_rank(self, n_user, n_item, n_sample, sample_item, accu, sample_topk):
        si, accu = _i32(sample_item), _i32(accu)
        out = np.empty(n_sample, np.int32)
        cost = np.zeros(1, np.int64)
        with self._tmp() as d:
            self.lib.ref_find_optimal_sample_rank(d.encode(), C.c_int64(n_user), C.c_int64(n_item),
                                                  C.c_int32(n_sample), _p(si), _p(accu), C.c_int32(si.shape[0]),
                                                  C.c_int32(sample_topk), _p(out), _p(cost))
        return out, int(cost[0])

    def uniform_sample_rank(self, n_item, n_sample):
        out = np.empty(n_sample, np.int32)
        self.lib.ref_uniform_sample_rank(C.c_int32(n_item), C.c_int32(n_sample), _p(out))
        return out

    def fit_regression(self, thr, n_item, sample_rank):
        thr, sr = _f32(thr), _i32(sample_rank)
        out = np.empty((thr.shape[0], 7), np.float32)
        with self._tmp() as d:
            rc = self.lib.ref_fit_regression(d.encode(), _p(thr), C.c_int64(thr.shape[0]), C.c_int64(n_item),
                                             _p(sr), C.c_int32(sr.shape[0]), _p(out))
        assert rc == 0
        return out

    def regression_rank_bound(self, reg, reg_rank, n_item, user_ids, qlb, qub):
        reg, rr = _f32(reg), _i32(reg_rank)
        ids, qlb, qub = _i32(user_ids), _f32(qlb), _f32(qub)
        lb = np.empty(ids.shape[0], np.int32)
        ub = np.empty(ids.shape[0], np.int32)
        with self._tmp() as d:
            self.lib.ref_regression_rank_bound(d.encode(), C.c_int64(reg.shape[0]), C.c_int64(n_item), _p(rr),
                                               C.c_int32(rr.shape[0]), _p(reg), C.c_int64(ids.shape[0]), _p(ids),
                                               _p(qlb), _p(qub), _p(lb), _p(ub))
        return lb, ub

    def svd_build(self, user, item, sigma=0.7):
        user, item = _f32(user), _f32(item)
        d = user.shape[1]
        ti = np.empty((d, d), np.float32)
        su = np.empty_like(user)
        cd = np.zeros(1, np.int32)
        self.lib.ref_svd_build(_p(user), C.c_int64(user.shape[0]), _p(item), C.c_int64(item.shape[0]),
                               C.c_int32(d), C.c_float(sigma), _p(ti), _p(su), _p(cd))
        return ti, su, int(cd[0])

    def qs_retrieval(self, user, item, check_dim, sample_rank, thr, query, topk):
        user, item, sr, thr, query = _f32(user), _f32(item), _i32(sample_rank), _f32(thr), _f32(query)
        nq = query.shape[0]
        out = np.zeros((nq, topk), USER_RANK)
        st = np.zeros(nq, STATS)
        with self._tmp() as d:
            self.lib.ref_qs_retrieval(d.encode(), _p(user), C.c_int64(user.shape[0]), _p(item),
                                      C.c_int64(item.shape[0]), C.c_int32(user.shape[1]), C.c_int32(check_dim),
                                      _p(sr), C.c_int32(sr.shape[0]), _p(thr), _p(query), C.c_int32(nq),
                                      C.c_int32(topk), C.c_int32(self.n_thread), _p(out), _p(st))
        return out, st

    def us_retrieval(self, user, item, sample_rank, thr, query, topk):
        user, item, sr, thr, query = _f32(user), _f32(item), _i32(sample_rank), _f32(thr), _f32(query)
        nq = query.shape[0]
        out = np.zeros((max(nq, 100), topk), USER_RANK)
        st = np.zeros(max(nq, 100), STATS)
        with self._tmp() as d:
            n = self.lib.ref_us_retrieval(d.encode(), _p(user), C.c_int64(user.shape[0]), _p(item),
                                          C.c_int64(item.shape[0]), C.c_int32(user.shape[1]), _p(sr),
                                          C.c_int32(sr.shape[0]), _p(thr), _p(query), C.c_int32(nq),
                                          C.c_int32(topk), C.c_int32(self.n_thread), _p(out), _p(st))
        return out[:n], st[:n]

    def qsrp_retrieval(self, user, svd_user, transfer_item, item, check_dim, sample_rank, thr, reg_rank, reg,
                       query, topk):
        user, svd_user, ti, item = _f32(user), _f32(svd_user), _f32(transfer_item), _f32(item)
        sr, thr, rr, reg, query = _i32(sample_rank), _f32(thr), _i32(reg_rank), _f32(reg), _f32(query)
        nq = query.shape[0]
        out = np.zeros((nq, topk), USER_RANK)
        st = np.zeros(nq, STATS)
        with self._tmp() as d:
            self.lib.ref_qsrp_retrieval(d.encode(), _p(user), _p(svd_user), _p(ti), C.c_int64(user.shape[0]),
                                        _p(item), C.c_int64(item.shape[0]), C.c_int32(user.shape[1]),
                                        C.c_int32(check_dim), _p(sr), C.c_int32(sr.shape[0]), _p(thr), _p(rr),
                                        _p(reg), _p(query), C.c_int32(nq), C.c_int32(topk),
                                        C.c_int32(self.n_thread), _p(out), _p(st))
        return out, st


class ReferenceQsrp:
    """The reference's QSRPNormalLP index held open for repeated Retrieval timing (oracle/_ref)."""

    def __init__(self, user, svd_user, transfer_item, item, check_dim, sample_rank, thr, reg_rank, reg, n_thread,
                 so=REF_SO):
        self.lib = C.CDLL(so)
        self.lib.ref_qsrp_open.restype = C.c_void_p
        self.lib.ref_set_threads(C.c_int(n_thread))
        self._keep = [_f32(user), _f32(svd_user), _f32(transfer_item), _f32(item), _i32(sample_rank), _f32(thr),
                      _i32(reg_rank), _f32(reg)]
        u, su, ti, it, sr, th, rr, rg = self._keep
        self.dir = tempfile.mkdtemp(prefix="rkr_ref_qsrp_")
        self.h = self.lib.ref_qsrp_open(self.dir.encode(), _p(u), _p(su), _p(ti), C.c_int64(u.shape[0]), _p(it),
                                        C.c_int64(it.shape[0]), C.c_int32(u.shape[1]), C.c_int32(check_dim), _p(sr),
                                        C.c_int32(sr.shape[0]), _p(th), _p(rr), _p(rg), C.c_int32(n_thread))
        self._keep = None

    def run(self, query, topk):
        q = _f32(query)
        out = np.zeros((q.shape[0], topk), USER_RANK)
        st = np.zeros(q.shape[0], STATS)
        secs = C.c_double()
        self.lib.ref_qsrp_run(C.c_void_p(self.h), _p(q), C.c_int32(q.shape[0]), C.c_int32(topk), _p(out), _p(st),
                              C.byref(secs))
        return out, st, secs.value

    def close(self):
        if self.h:
            self.lib.ref_qsrp_close(C.c_void_p(self.h))
            self.h = None
