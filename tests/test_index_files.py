"""The reference's on-disk index formats (rkr_file_*), on the CPU.

Files written by the reference's own writers (oracle/_ref: SampleSearch::SaveIndex,
NormalLinearRegressionLP::SaveIndex, WriteDistributionBelowTopk) must read back through the engine's
readers to the arrays that produced them, and the engine's writers must produce the same bytes.
The SVD layout (SVD::SaveIndex, which needs Armadillo in the reference) is checked by its size,
header and a round trip.  Damaged files are RKR_ERR_IO.
"""
import ctypes as C
import os

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle, Reference

needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.fixture(scope="module")
def data():
    orc = Oracle()
    rng = np.random.default_rng(77)
    n_user, n_item, d = 300, 900, 16
    user = orc.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * 2).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, 10), np.linspace(10, n_item - 2, 22).astype(int)])).astype(np.int32)
    thr = orc.build_thresholds(user, item, rank)
    return dict(orc=orc, user=user, item=item, rank=rank, thr=thr, n_user=n_user, n_item=n_item, d=d)


@needs_ref
@pytest.mark.parametrize("query_distribution", [True, False])
def test_sample_search_file_matches_the_reference_writer(data, tmp_path, query_distribution):
    ref = Reference()
    S = data["rank"].shape[0]
    ref.lib.ref_write_sample_search(str(tmp_path).encode(), b"ds", b"QS" if query_distribution else b"US",
                                    _p(data["rank"]), C.c_int32(S), _p(data["thr"]), C.c_int64(data["n_user"]),
                                    C.c_int64(data["n_item"]), C.c_int32(7), C.c_int32(3),
                                    C.c_int32(int(query_distribution)))
    name = f"QS-ds-n_sample_{S}-n_sample_query_7-sample_topk_3.index" if query_distribution else f"US-ds-n_sample_{S}.index"
    path = tmp_path / "memory_index" / name
    rank, thr, n_item = R.read_sample_search(path)
    assert n_item == data["n_item"]
    assert np.array_equal(rank, data["rank"])
    assert np.array_equal(thr.view(np.int32), data["thr"].view(np.int32))
    mine = tmp_path / "mine.index"
    R.write_sample_search(mine, data["rank"], data["n_item"], data["thr"])
    assert mine.read_bytes() == path.read_bytes()
    # the ranks-only form (qrs_to_sample_index)
    R.write_sample_search(tmp_path / "ranks.index", data["rank"], data["n_item"], None, n_user=data["n_user"])
    r2, t2, _ = R.read_sample_search(tmp_path / "ranks.index")
    assert np.array_equal(r2, data["rank"]) and t2 is None
    assert (tmp_path / "ranks.index").read_bytes() == path.read_bytes()[:24 + 4 * S]


@needs_ref
def test_regression_file_matches_the_reference_writer(data, tmp_path):
    ref = Reference()
    S = data["rank"].shape[0]
    rec = np.empty((data["n_user"], 7), np.float32)
    rc = ref.lib.ref_fit_regression(str(tmp_path).encode(), _p(data["thr"]), C.c_int64(data["n_user"]),
                                    C.c_int64(data["n_item"]), _p(data["rank"]), C.c_int32(S), _p(rec))
    assert rc == 0
    path = tmp_path / "memory_index" / f"NormalLinearRegressionLP-QS-h-n_sample_{S}-n_sample_query_0-sample_topk_0.index"
    rank, got, n_item = R.read_regression(path)
    assert n_item == data["n_item"] and np.array_equal(rank, data["rank"])
    assert np.array_equal(got.view(np.int32), rec.view(np.int32))
    mine = tmp_path / "mine.index"
    R.write_regression(mine, data["rank"], rec, data["n_item"])
    assert mine.read_bytes() == path.read_bytes()


@needs_ref
def test_query_distribution_matches_the_reference_writer(data, tmp_path):
    ref = Reference()
    n_s, topk = 40, 12
    si = ref.sample_item(data["n_item"], n_s)
    accu = ref.query_rank_distribution(data["user"], data["item"], si)
    kth, sid = ref.sort_kth_rank(accu, topk)
    ref.lib.ref_write_query_distribution(str(tmp_path).encode(), b"ds", _p(si), _p(kth), _p(sid), _p(accu),
                                         C.c_int64(data["n_item"]), C.c_int32(n_s), C.c_int32(topk))
    rdir = tmp_path / "query_distribution" / f"ds-n_sample_item_{n_s}-sample_topk_{topk}"
    mdir = tmp_path / "mine"
    R.write_query_distribution(mdir, si, kth, sid, accu)
    for f in ("sample_itemID_l.txt", "sort_kth_rank_l.index", "accu_n_user_rank_l.index"):
        assert (mdir / f).read_bytes() == (rdir / f).read_bytes(), f
    s2, k2, a2 = R.read_query_distribution(rdir, n_s, data["n_item"])
    assert np.array_equal(s2, si[sid]) and np.array_equal(k2, kth) and np.array_equal(a2, accu[sid])


def test_svd_file_round_trip_and_layout(data, tmp_path):
    ti, su, cd = R.svd_build(data["user"], 0.7)
    path = tmp_path / "svd_index" / "ds.index"
    path.parent.mkdir()
    R.write_svd(path, ti, su, cd, data["n_item"])
    n, d, ni = data["n_user"], data["d"], data["n_item"]
    raw = path.read_bytes()
    assert len(raw) == 32 + 4 * d * (d + n + ni)
    assert np.frombuffer(raw[:24], np.uint64).tolist() == [n, ni, d]
    assert np.frombuffer(raw[24:28], np.float32)[0] == np.float32(0.7)
    assert np.frombuffer(raw[28:32], np.int32)[0] == cd
    got = R.read_svd(path, with_items=True)
    assert got["check_dim"] == cd and got["n_item"] == ni
    assert np.array_equal(got["transfer_item"], ti) and np.array_equal(got["svd_user"], su)
    assert not got["svd_item"].any()


def test_damaged_files_are_io_errors(data, tmp_path):
    p = tmp_path / "x.index"
    R.write_sample_search(p, data["rank"], data["n_item"], data["thr"])
    raw = p.read_bytes()
    for bad in (raw[:-4], raw[:10], raw + b"\0"):
        p.write_bytes(bad)
        with pytest.raises(R.RkrError) as e:
            R.read_sample_search(p)
        assert e.value.status == R.RKR_ERR_IO
    with pytest.raises(R.RkrError) as e:
        R.read_regression(tmp_path / "missing.index")
    assert e.value.status == R.RKR_ERR_IO
    q = tmp_path / "r.index"
    R.write_regression(q, data["rank"], np.zeros((data["n_user"], 7), np.float32), data["n_item"])
    q.write_bytes(q.read_bytes()[:-1])
    with pytest.raises(R.RkrError) as e:
        R.read_regression(q)
    assert e.value.status == R.RKR_ERR_IO
    with pytest.raises(R.RkrError) as e:
        R.read_svd(q)
    assert e.value.status == R.RKR_ERR_IO
