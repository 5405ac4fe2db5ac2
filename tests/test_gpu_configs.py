"""GPU parity on the reference's own dataset and on the CPU-runnable workload.

* refdataset: the reference's bundled dataset (dataset/fake-normal-30d: 1,000 users, 5,000 items,
  100 queries, d = 30) through the reference's pipeline with its driver script's parameters
  (run_rkr.py:73-78,104: 150 sampled items, sample_topk 40, 20 sampled ranks, k in {10, 20, 30}).
  The expected values are the reference's own outputs (tests/golden/refdataset.npz, made by
  tests/golden/make_golden.py from oracle/_ref).
* config 1: 1,000 users x 5,000 items, d = 30, entries i.i.d. N(0, 1) drawn in FP64, 64 sampled
  thresholds per user (OptimalPart ranks over 150 sampled items), 100 queries drawn from the items,
  k = 10: the whole index built through the C ABI, then QS / QSRPNormalLP / US against the oracle.
All comparisons are bit for bit: ids, ranks, the binary32 patterns of reported scores and counters.
"""
import os

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle, Reference, ReferenceQsrp

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STATS = ("n_prune", "n_result", "n_refine", "ip_cost")


def same(a, b):
    a = np.ascontiguousarray(a).view(np.int32).reshape(-1)
    b = np.ascontiguousarray(b).view(np.int32).reshape(-1)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.fixture(scope="module")
def ref_ds():
    return dict(np.load(os.path.join(GOLDEN, "refdataset.npz")))


def test_refdataset_build_matches_reference(ref_ds):
    g = ref_ds
    assert same(R.normalize(g["user"]), g["user_norm"])
    with R.Index(g["user_norm"], g["item"]) as ix:
        assert np.array_equal(ix.query_rank_distribution(g["sample_item"]), g["accu"])
        assert same(ix.build_sample_search(g["uni_rank"]), g["thr_uni"])
        assert same(ix.build_sample_search(g["opt_rank"]), g["thr"])
    kth, sid = R.sort_kth_rank(g["accu"], int(g["sample_topk"]))
    rank, cost = R.find_optimal_sample_rank(g["user"].shape[0], g["item"].shape[0], 20, kth, g["accu"][sid])
    assert np.array_equal(rank, g["opt_rank"]) and cost == int(g["opt_cost"])


@pytest.mark.parametrize("k", [10, 20, 30])
def test_refdataset_queries_match_reference(ref_ds, k):
    """Each k from a fresh index, as each of the driver's rri runs is."""
    g = ref_ds
    cd = int(g["check_dim"])
    with R.Index(g["user_norm"], g["item"]) as ix:
        ix.load_sample_search(g["opt_rank"], g["thr"])
        ix.load_svd(cd, g["transfer_item"], g["svd_user"])
        ix.load_regression(g["opt_rank"], g["reg"])
        out, st = ix.retrieval("QS", g["query"], k, stats=True)
        assert same(out, g[f"qs_{k}"])
        for f in STATS:
            assert np.array_equal(st[f], g[f"qs_stats_{k}"][f]), ("QS", f)
        out, st = ix.retrieval("QSRPNormalLP", g["query"], k, stats=True)
        assert same(out, g[f"qsrp_{k}"])
        for f in STATS:
            assert np.array_equal(st[f], g[f"qsrp_stats_{k}"][f]), ("QSRP", f)
    with R.Index(g["user_norm"], g["item"]) as ix:
        ix.load_sample_search(g["uni_rank"], g["thr_uni"])
        out, st = ix.retrieval("US", g["query"], k, stats=True)
        assert same(out, g[f"us_{k}"])
        for f in ("n_refine", "ip_cost"):
            assert np.array_equal(st[f], g[f"us_stats_{k}"][f]), ("US", f)


def test_config1_whole_pipeline_matches_oracle():
    """The CPU-runnable workload: every stage through the C ABI, then the three methods."""
    n_user, n_item, d, n_sample, n_si, stopk, nq, k = 1000, 5000, 30, 64, 150, 10, 100, 10
    rng = np.random.default_rng(1)
    user = rng.standard_normal((n_user, d)).astype(np.float32)   # drawn in FP64, stored as fvecs FP32
    item = np.random.default_rng(2).standard_normal((n_item, d)).astype(np.float32)
    query = item[np.random.default_rng(3).choice(n_item, nq, replace=False)].copy()
    orc = Oracle()
    un = R.normalize(user)
    assert same(un, orc.normalize(user))
    si = R.sample_item(n_item, n_si)
    with R.Index(un, item) as ix:
        accu = ix.query_rank_distribution(si)
        _, accu_o = orc.query_rank_distribution(un, item, si)
        assert np.array_equal(accu, accu_o)
        kth, sid = R.sort_kth_rank(accu, stopk)
        rank, _ = R.find_optimal_sample_rank(n_user, n_item, n_sample, kth, accu[sid])
        assert np.array_equal(rank, orc.optimal_sample_rank(n_user, n_item, n_sample, kth, accu[sid])[0])
        thr = ix.build_sample_search(rank)
        assert same(thr, orc.build_thresholds(un, item, rank))
        reg = R.fit_regression(thr)
        ti, su, cd = R.svd_build(un, 0.7)
        ix.load_svd(cd, ti, su)
        ix.load_regression(rank, reg)
        a, sa = ix.retrieval("QS", query, k, stats=True)
        b, sb = orc.qs_retrieval(un, item, cd, rank, thr, query, k)
        assert same(a, b)
        for f in STATS:
            assert np.array_equal(sa[f], sb[f]), ("QS", f)
        a, sa = ix.retrieval("QSRPNormalLP", query, k, stats=True)
        b, sb = orc.qsrp_retrieval(un, su, ti, item, cd, rank, thr, rank, reg, query, k)
        assert same(a, b)
        for f in STATS:
            assert np.array_equal(sa[f], sb[f]), ("QSRP", f)
        if Reference.available():
            ref = ReferenceQsrp(un, su, ti, item, cd, rank, thr, rank, reg, os.cpu_count() or 1)
            try:
                c, _, _ = ref.run(query, k)
            finally:
                ref.close()
            assert same(a, c)
    uni = R.uniform_sample_rank(n_item, n_sample)
    with R.Index(un, item) as ix:
        thr_u = ix.build_sample_search(uni)
        a = ix.retrieval("US", query, k)
        b, _ = orc.us_retrieval(un, item, uni, thr_u, query, k)
        assert same(a, b)


@pytest.mark.parametrize("n_item", [40000, 90001])
def test_build_rows_larger_than_shared_memory_match_oracle(n_item):
    """Rows too long for the shared-memory selection (config 4 has 624,961 items) take the
    global-memory path of the row selection: thresholds (a dense head of ranks, then a spread) and
    the query-rank distribution against the oracle, with lognormal item norms as at config 4."""
    n_user, d = 192, 24
    rng = np.random.default_rng(n_item)
    orc = Oracle()
    user = orc.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, 64), np.linspace(64, n_item - 2, 200).astype(int)])).astype(np.int32)
    si = R.sample_item(n_item, 40)
    with R.Index(user, item) as ix:
        thr = ix.build_sample_search(rank)
        assert same(thr, orc.build_thresholds(user, item, rank))
        accu = ix.query_rank_distribution(si)
        _, accu_o = orc.query_rank_distribution(user, item, si)
        assert np.array_equal(accu, accu_o)


@pytest.mark.parametrize("n_item", [3001, 40003])
def test_query_rank_distribution_with_equal_scores_matches_oracle(n_item):
    """Items drawn from 50 distinct vectors (every score repeated), rows of both lengths (shared-memory
    and longer), an item count that is not a multiple of four: the counting of items strictly above
    each sampled item's score, and the thresholds (requested bins far larger than the staging buffer),
    against the oracle."""
    n_user, d = 300, 16
    rng = np.random.default_rng(n_item + 7)
    orc = Oracle()
    user = orc.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    base = rng.standard_normal((50, d)).astype(np.float32)
    item = base[rng.integers(0, 50, n_item)]
    si = R.sample_item(n_item, 150)
    rank = np.unique(np.concatenate([np.arange(0, 40), np.linspace(40, n_item - 2, 200).astype(int)])).astype(np.int32)
    with R.Index(user, item) as ix:
        accu = ix.query_rank_distribution(si)
        thr = ix.build_sample_search(rank)
    _, accu_o = orc.query_rank_distribution(user, item, si)
    assert np.array_equal(accu, accu_o)
    assert same(thr, orc.build_thresholds(user, item, rank))
