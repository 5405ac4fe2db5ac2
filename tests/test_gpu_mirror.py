"""The C++ BaseIndex mirror (reverse-k-ranks_b200/host/B200Index.hpp) linked and run inside the
reference's query app, on index files the reference's own writers produced.

oracle/_ref/rri_b200 (built by `make -C oracle ref` from the reference's headers and
oracle/rri_b200.cpp) reads a dataset with the reference's readData, builds the reference's own
QS / QSRPNormalLP / US index from the index files and the B200 mirror of it, answers the query file
with both and writes both through the reference's WriteRankResult.  The index files come from the
reference harness (oracle/_ref/librkr_ref.so): the sampled-threshold index through the reference's
SampleSearch::SaveIndex, the SVD and regression files in the layouts their LoadIndex reads.  The
userID, rank and IP CSV files of the two runs must be identical byte for byte.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import rkr_b200 as R
from checkers import REF_SO, ROOT, USER_RANK, STATS, Oracle, Reference

pytestmark = pytest.mark.gpu

RRI = os.path.join(ROOT, "oracle", "_ref", "rri_b200")


def write_fvecs(path, a):
    a = np.ascontiguousarray(a, np.float32)
    rows = np.empty((a.shape[0], a.shape[1] + 1), np.int32)
    rows[:, 0] = a.shape[1]
    rows[:, 1:] = a.view(np.int32)
    rows.tofile(path)


@pytest.mark.skipif(not (os.path.exists(RRI) and Reference.available()), reason="oracle/_ref not built")
def test_mirror_app_writes_the_reference_apps_results(tmp_path):
    orc = Oracle()
    rng = np.random.default_rng(31)
    n_user, n_item, d, nq, S, topk = 700, 1600, 24, 100, 32, 10
    user = (rng.standard_normal((n_user, d)) * 2).astype(np.float32)
    item = (rng.standard_normal((n_item, d)) * 2).astype(np.float32)
    query = np.concatenate([item[rng.choice(n_item, nq // 2, replace=False)],
                            (rng.standard_normal((nq - nq // 2, d)) * 2).astype(np.float32)])
    data = tmp_path / "data" / "h"
    data.mkdir(parents=True)
    write_fvecs(data / "h_user.fvecs", user)
    write_fvecs(data / "h_data_item.fvecs", item)
    write_fvecs(data / "h_query_item.fvecs", query)
    un = orc.normalize(user)  # what readData leaves (VectorIO.hpp:61)
    rank = np.unique(np.concatenate([np.arange(0, 12), np.linspace(12, n_item - 2, S - 12).astype(int)]))
    rank = rank.astype(np.int32)
    S = rank.shape[0]
    uni = orc.uniform_sample_rank(n_item, S)
    thr, thr_uni = orc.build_thresholds(un, item, rank), orc.build_thresholds(un, item, uni)
    reg = orc.fit_regression(thr)
    ti, su, cd = R.svd_build(un, 0.7)
    index = tmp_path / "index"
    index.mkdir()
    # the reference harness writes the index files (and answers once, which is not used here)
    lib = C.CDLL(REF_SO)
    p = lambda a: np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)
    out = np.zeros((nq, topk), USER_RANK)
    st = np.zeros(nq, STATS)
    lib.ref_qsrp_retrieval(str(index).encode(), p(un), p(su), p(ti), C.c_int64(n_user), p(item), C.c_int64(n_item),
                           C.c_int32(d), C.c_int32(cd), p(rank), C.c_int32(S), p(thr), p(rank), p(reg), p(query),
                           C.c_int32(nq), C.c_int32(topk), C.c_int32(1), p(out), p(st))
    lib.ref_us_retrieval(str(index).encode(), p(un), C.c_int64(n_user), p(item), C.c_int64(n_item), C.c_int32(d),
                         p(uni), C.c_int32(S), p(thr_uni), p(query), C.c_int32(nq), C.c_int32(topk), C.c_int32(1),
                         p(out), p(st))
    (tmp_path / "bin").mkdir()
    (tmp_path / "result" / "rank").mkdir(parents=True)
    for method, nsq, stopk in (("QS", 1, 1), ("QSRPNormalLP", 1, 1), ("US", 0, 0)):
        r = subprocess.run([RRI, str(tmp_path / "data"), "h", str(index), method, str(topk), str(S), str(nsq),
                            str(stopk)], cwd=tmp_path / "bin", capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        for part in ("userID", "rank", "IP"):
            a = (tmp_path / "result" / "rank" / f"h-{method}-ref-{part}.csv").read_bytes()
            b = (tmp_path / "result" / "rank" / f"h-{method}-b200-{part}.csv").read_bytes()
            assert len(a) > 0 and a == b, (method, part)


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")
def test_index_load_files_answers_as_the_explicit_loads(tmp_path):
    """rkr_index_load_files on the files the reference's writers produced answers every method exactly
    as an index loaded array by array; a file of another user count is refused."""
    orc = Oracle()
    rng = np.random.default_rng(32)
    n_user, n_item, d, nq, topk = 500, 1200, 20, 100, 10  # US answers 100 queries per call
    user = orc.normalize((rng.standard_normal((n_user, d)) * 2).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * 2).astype(np.float32)
    query = item[rng.choice(n_item, nq, replace=False)].copy()
    rank = np.unique(np.linspace(0, n_item - 2, 30).astype(np.int32))
    S = rank.shape[0]
    thr = orc.build_thresholds(user, item, rank)
    ti, su, cd = R.svd_build(user, 0.7)
    ref = Reference()
    p = lambda a: np.ascontiguousarray(a).ctypes.data_as(C.c_void_p)
    rec = np.empty((n_user, 7), np.float32)
    assert ref.lib.ref_fit_regression(str(tmp_path).encode(), p(thr), C.c_int64(n_user), C.c_int64(n_item), p(rank),
                                      C.c_int32(S), p(rec)) == 0
    for name, qd in ((b"QS", 1), (b"US", 0)):
        ref.lib.ref_write_sample_search(str(tmp_path).encode(), b"h", name, p(rank), C.c_int32(S), p(thr),
                                        C.c_int64(n_user), C.c_int64(n_item), C.c_int32(0), C.c_int32(0), C.c_int32(qd))
    R.write_svd(tmp_path / "svd_index" / "h.index", ti, su, cd, n_item)
    for method in ("QS", "QSRPNormalLP", "US"):
        with R.Index(user, item) as a, R.Index(user, item) as b:
            a.load_files(method, str(tmp_path), "h", S, 0, 0)
            b.load_sample_search(rank, thr)
            if method != "US":
                b.load_svd(cd, ti, su) if method == "QSRPNormalLP" else b.set_check_dim(cd)
            if method == "QSRPNormalLP":
                b.load_regression(rank, rec)
            ra = a.retrieval(method, query, topk)
            rb = b.retrieval(method, query, topk)
            assert np.array_equal(ra.view(np.int32), rb.view(np.int32)), method
    with R.Index(user[:-1], item) as c:
        with pytest.raises(R.RkrError) as e:
            c.load_files("QS", str(tmp_path), "h", S, 0, 0)
        assert e.value.status == R.RKR_ERR_IO
