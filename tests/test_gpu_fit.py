"""The regression fit on the device (rkr_index_fit_regression) against the host fit (rkr_fit_regression,
the same arithmetic) bit for bit, and against the reference's own records (tests/golden) as the host
fit is checked in tests/test_abi.py: mu, sigma and the extremes bit-exact, (a, b, error) to the LP's
rounding (the reference's LP solver is randomised)."""
import os

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(case):
    return dict(np.load(os.path.join(GOLDEN, case + ".npz")))


def bits(a):
    return np.ascontiguousarray(a).view(np.int32)


@pytest.mark.parametrize("case", ["small", "fakenormal", "refdataset"])
def test_device_fit_matches_host_and_reference(case):
    g = load(case)
    with R.Index(g["user_norm"], g["item"]) as ix:
        ix.load_sample_search(g["opt_rank"], g["thr"])
        rec = ix.fit_regression()
    host = R.fit_regression(g["thr"])
    assert np.array_equal(bits(rec), bits(host))
    ref = g["reg"]
    assert np.array_equal(bits(rec[:, 2:4]), bits(ref[:, 2:4]))
    assert np.array_equal(bits(rec[:, 5:7]), bits(ref[:, 5:7]))
    np.testing.assert_allclose(rec[:, 4], ref[:, 4], rtol=1e-5, atol=1e-4)
    np.testing.assert_allclose(rec[:, :2], ref[:, :2], rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("n_sample", [20, 64, 512, 1500])
def test_device_fit_at_scale_matches_host(n_sample):
    rng = np.random.default_rng(n_sample)
    n_user, n_item, d = 30000, 4000, 48
    user = R.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.linspace(0, n_item - 1, n_sample).astype(np.int32))
    with R.Index(user, item) as ix:
        thr = ix.build_sample_search(rank)
        rec = ix.fit_regression()
    host = R.fit_regression(thr)
    diff = np.nonzero(np.any(bits(rec) != bits(host), axis=1))[0]
    assert diff.size == 0, (diff[:5], rec[diff[:3]], host[diff[:3]])


def test_queries_on_the_device_fit_match_the_oracle():
    orc = Oracle()
    rng = np.random.default_rng(9)
    n_user, n_item, d = 6000, 3000, 40
    user = R.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, 20), np.linspace(20, n_item - 2, 44).astype(int)])).astype(np.int32)
    query = item[rng.choice(n_item, 40, replace=False)].copy()
    ti, su, cd = R.svd_build(user, 0.7)
    with R.Index(user, item) as ix:
        thr = ix.build_sample_search(rank)
        reg = ix.fit_regression()
        ix.load_svd(cd, ti, su)
        out = ix.retrieval("QSRPNormalLP", query, 25)
    want, _ = orc.qsrp_retrieval(user, su, ti, item, cd, rank, thr, rank, reg, query, 25)
    assert np.array_equal(bits(out).reshape(-1), bits(want).reshape(-1))


def test_device_fit_needs_thresholds():
    rng = np.random.default_rng(1)
    with R.Index(rng.standard_normal((100, 8)).astype(np.float32), rng.standard_normal((50, 8)).astype(np.float32)) as ix:
        with pytest.raises(R.RkrError):
            ix.fit_regression()


@pytest.mark.parametrize("case", ["small", "refdataset"])
def test_device_svd_is_the_host_transform_to_rounding(case):
    """rkr_index_svd_build: a valid transform (transfer_user . (transfer_item q) == <user, q>), the
    host build's check_dim, and its matrices to the rounding of the Gram matrix's other summation
    order; queries on it answer as the oracle does on the same SVD index."""
    g = load(case)
    un = g["user_norm"]
    with R.Index(un, g["item"]) as ix:
        ti, su, cd = ix.svd_build(0.7)
        ix.load_sample_search(g["opt_rank"], g["thr"])
        ix.load_regression(g["opt_rank"], g["reg"])
        k = 10
        out = ix.retrieval("QSRPNormalLP", g["query"], k)
    with R.Index(un, g["item"]) as ix2:  # the same transform on every run
        ti2, su2, cd2 = ix2.svd_build(0.7)
    assert np.array_equal(bits(ti2), bits(ti)) and np.array_equal(bits(su2), bits(su)) and cd2 == cd
    hti, hsu, hcd = R.svd_build(un, 0.7)
    assert cd == hcd
    q = g["query"][:8].astype(np.float64)
    np.testing.assert_allclose(su.astype(np.float64) @ (ti.astype(np.float64) @ q.T), un.astype(np.float64) @ q.T,
                               atol=2e-4)
    np.testing.assert_allclose(ti, hti, atol=2e-5)
    np.testing.assert_allclose(su, hsu, atol=2e-5)
    want, _ = Oracle().qsrp_retrieval(un, su, ti, g["item"], cd, g["opt_rank"], g["thr"], g["opt_rank"], g["reg"],
                                      g["query"], k)
    assert np.array_equal(bits(out).reshape(-1), bits(want).reshape(-1))


def test_score_table_file_matches_the_oracle(tmp_path):
    """rkr_file_write_score_table: bstb's table (descending score rows, no header) for the first users."""
    g = load("small")
    n_out, n_item = 120, g["item"].shape[0]
    path = tmp_path / "small.index"
    with R.Index(g["user_norm"], g["item"]) as ix:
        ix.write_score_table(str(path), n_out)
        with pytest.raises(R.RkrError):
            ix.write_score_table(str(tmp_path / "too_many.index"), ix.n_user + 1)
    rows = np.fromfile(path, np.float32)
    assert rows.size == n_out * n_item
    want = Oracle().score_sort_rows(g["user_norm"], g["item"], 0, n_out)
    assert np.array_equal(bits(rows), bits(want).reshape(-1))
