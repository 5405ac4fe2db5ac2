"""Pins the oracle (oracle/rkr_oracle.c) against the reference's own code.

* Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from oracle/_ref, the
  reference's headers compiled unmodified) -- run everywhere.
* Live comparison with oracle/_ref on fresh seeded inputs and on the reference's bundled
  fake-normal-30d dataset -- run where the harness was built.
All comparisons are bit-exact (float results compared as bit patterns).
"""
import os

import numpy as np
import pytest

from checkers import Oracle, Reference, USER_RANK, reference_root

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["small", "fakenormal"]
REF_DATASET = os.path.join(reference_root(), "dataset", "fake-normal-30d", "fake-normal-30d")


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def bits(a):
    return np.ascontiguousarray(a).view(np.int32)


def same_results(a, b):
    return np.array_equal(bits(np.ascontiguousarray(a)).reshape(-1), bits(np.ascontiguousarray(b)).reshape(-1))


@pytest.mark.parametrize("case", CASES)
def test_build_stages_match_golden(orc, case):
    g = load(case)
    un = orc.normalize(g["user"])
    assert np.array_equal(bits(un), bits(g["user_norm"]))
    ranks, accu = orc.query_rank_distribution(un, g["item"], g["sample_item"])
    assert np.array_equal(accu, g["accu"])
    assert (accu[:, -1] == un.shape[0]).all()  # QueryRankByComputation.hpp:238
    kth = orc.kth_rank(accu, int(g["sample_topk"]))
    assert np.array_equal(np.sort(kth), g["sort_kth"])
    assert np.array_equal(kth[g["sort_sid"]], g["sort_kth"])
    opt, cost = orc.optimal_sample_rank(un.shape[0], g["item"].shape[0], g["opt_rank"].shape[0], g["sort_kth"],
                                        g["accu"][g["sort_sid"]])
    assert np.array_equal(opt, g["opt_rank"])
    assert cost == int(g["opt_cost"])
    assert np.array_equal(orc.uniform_sample_rank(g["item"].shape[0], g["uni_rank"].shape[0]), g["uni_rank"])
    thr = orc.build_thresholds(un, g["item"], g["opt_rank"])
    assert np.array_equal(bits(thr), bits(g["thr"]))
    assert (np.diff(thr, axis=1) <= 0).all()
    reg = orc.fit_regression(g["thr"])
    assert np.array_equal(bits(reg), bits(g["reg"]))


@pytest.mark.parametrize("case", CASES)
def test_query_methods_match_golden(orc, case):
    g = load(case)
    k = int(g["topk"])
    qs, st = orc.qs_retrieval(g["user_norm"], g["item"], int(g["check_dim"]), g["opt_rank"], g["thr"], g["query"], k)
    assert same_results(qs, g["qs"])
    assert np.array_equal(st["n_refine"], g["qs_stats"]["n_refine"])
    assert np.array_equal(st["n_prune"], g["qs_stats"]["n_prune"])
    assert np.array_equal(st["ip_cost"], g["qs_stats"]["ip_cost"])
    qsrp, st = orc.qsrp_retrieval(g["user_norm"], g["svd_user"], g["transfer_item"], g["item"], int(g["check_dim"]),
                                  g["opt_rank"], g["thr"], g["opt_rank"], g["reg"], g["query"], k)
    assert same_results(qsrp, g["qsrp"])
    assert np.array_equal(st["n_result"], g["qsrp_stats"]["n_result"])
    assert np.array_equal(st["ip_cost"], g["qsrp_stats"]["ip_cost"])
    q100 = np.concatenate([g["query"]] * (100 // g["query"].shape[0] + 1))[:100]
    us, st = orc.us_retrieval(g["user_norm"], g["item"], g["uni_rank"], g["thr_uni"], q100, k)
    assert same_results(us, g["us"])
    assert np.array_equal(st["ip_cost"], g["us_stats"]["ip_cost"])


def test_oracle_matches_reference_dataset_golden(orc):
    """The reference's bundled dataset (dataset/fake-normal-30d) with its driver's parameters
    (run_rkr.py:73-78,104), every build stage and QS / QSRPNormalLP / US at k = 10, 20, 30, each k from a
    fresh index: the oracle equals the reference's outputs stored in tests/golden/refdataset.npz."""
    g = load("refdataset")
    un = orc.normalize(g["user"])
    assert np.array_equal(bits(un), bits(g["user_norm"]))
    n_user, n_item = un.shape[0], g["item"].shape[0]
    _, accu = orc.query_rank_distribution(un, g["item"], g["sample_item"])
    assert np.array_equal(accu, g["accu"])
    kth = orc.kth_rank(accu, int(g["sample_topk"]))
    sid = np.argsort(kth, kind="stable")
    opt, cost = orc.optimal_sample_rank(n_user, n_item, g["opt_rank"].shape[0], kth[sid], accu[sid])
    assert np.array_equal(opt, g["opt_rank"]) and cost == int(g["opt_cost"])
    assert np.array_equal(orc.uniform_sample_rank(n_item, g["uni_rank"].shape[0]), g["uni_rank"])
    assert np.array_equal(bits(orc.build_thresholds(un, g["item"], g["opt_rank"])), bits(g["thr"]))
    assert np.array_equal(bits(orc.build_thresholds(un, g["item"], g["uni_rank"])), bits(g["thr_uni"]))
    cd = int(g["check_dim"])
    for k in g["topks"]:
        qs, st = orc.qs_retrieval(un, g["item"], cd, g["opt_rank"], g["thr"], g["query"], int(k))
        assert same_results(qs, g[f"qs_{k}"])
        assert np.array_equal(st["ip_cost"], g[f"qs_stats_{k}"]["ip_cost"])
        qsrp, st = orc.qsrp_retrieval(un, g["svd_user"], g["transfer_item"], g["item"], cd, g["opt_rank"], g["thr"],
                                      g["opt_rank"], g["reg"], g["query"], int(k))
        assert same_results(qsrp, g[f"qsrp_{k}"])
        assert np.array_equal(st["n_result"], g[f"qsrp_stats_{k}"]["n_result"])
        us, st = orc.us_retrieval(un, g["item"], g["uni_rank"], g["thr_uni"], g["query"], int(k))
        assert same_results(us, g[f"us_{k}"])
        assert np.array_equal(st["ip_cost"], g[f"us_stats_{k}"]["ip_cost"])


@pytest.mark.parametrize("case", CASES)
def test_golden_ranks_are_bounded_by_exact_ranks(orc, case):
    """Reported QS ranks: refined users carry their exact rank, bound-accepted users rank_lb >= exact."""
    g = load(case)
    exact = orc.exact_rank_f64(g["user_norm"], g["item"], g["query"])
    qs = g["qs"]
    for q in range(qs.shape[0]):
        for e in qs[q]:
            assert e["rank"] >= exact[q, e["user_id"]] - 1  # FP32 vs FP64 ties may move one item


def test_sample_search_bounds_are_valid(orc):
    """rank_ub <= #{items >= q} <= rank_lb for every user and query (SampleSearch.hpp:110,127-129)."""
    rng = np.random.default_rng(5)
    user = orc.normalize(rng.standard_normal((60, 12)).astype(np.float32))
    item = rng.standard_normal((500, 12)).astype(np.float32)
    rank = np.array([0, 1, 2, 5, 9, 20, 40, 80, 160, 320, 499], np.int32)
    thr = orc.build_thresholds(user, item, rank)
    import ctypes as C
    for u in range(user.shape[0]):
        scores = np.array([orc.inner_product(user[u], it) for it in item], np.float32)
        for qv in rng.standard_normal((20, 12)).astype(np.float32):
            q = np.float32(orc.inner_product(qv, user[u]))
            lb, ub = C.c_int32(), C.c_int32()
            orc.lib.orc_sample_search_bound(thr[u].ctypes.data_as(C.c_void_p), C.c_int32(len(rank)),
                                            rank.ctypes.data_as(C.c_void_p), C.c_int64(item.shape[0]),
                                            C.c_float(q), C.byref(lb), C.byref(ub))
            n_ge = int((scores >= q).sum())
            assert ub.value <= n_ge <= lb.value


def test_regression_error_covers_fitted_points(orc):
    """The fitted line's error e bounds |a x + b - y| at every sample point (NormalLinearRegressionLP.hpp:241)."""
    g = load("fakenormal")
    reg = orc.fit_regression(g["thr"])
    S = g["thr"].shape[1]
    for u in range(0, reg.shape[0], 7):
        a, b, mu, sigma, err = (float(v) for v in reg[u, :5])
        assert 0 < err <= S + 0.1
        for j in range(S - 1):
            for x in (orc.cdf_phi((g["thr"][u, j] - mu) / sigma), orc.cdf_phi((g["thr"][u, j + 1] - mu) / sigma)):
                assert abs(a * float(x) + b - (j + 1)) <= err + 1e-3


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_oracle_matches_reference_on_fresh_inputs(orc):
    R = Reference(n_thread=2)
    rng = np.random.default_rng(2024)
    user = rng.standard_normal((200, 24)).astype(np.float32)
    item = rng.standard_normal((600, 24)).astype(np.float32)
    query = np.concatenate([item[:10], rng.standard_normal((10, 24)).astype(np.float32)])
    un = R.normalize(user)
    assert np.array_equal(bits(un), bits(orc.normalize(user)))
    rank = R.uniform_sample_rank(600, 24)
    thr = R.build_thresholds(un, item, rank)
    assert np.array_equal(bits(thr), bits(orc.build_thresholds(un, item, rank)))
    x = np.linspace(-7, 7, 20001).astype(np.float32)
    import ctypes as C
    r = np.empty_like(x)
    R.lib.ref_cdf_phi(x.ctypes.data_as(C.c_void_p), C.c_int64(len(x)), r.ctypes.data_as(C.c_void_p))
    o = np.array([orc.cdf_phi(v) for v in x], np.float32)
    assert np.array_equal(bits(r), bits(o))
    reg = R.fit_regression(thr, 600, rank)
    assert np.array_equal(bits(reg), bits(orc.fit_regression(thr)))
    ids = rng.integers(0, 200, 3000).astype(np.int32)
    qlb = rng.normal(0, 1.5, 3000).astype(np.float32)
    qub = (qlb + np.abs(rng.normal(0, 0.3, 3000))).astype(np.float32)
    assert all(np.array_equal(a, b) for a, b in zip(R.regression_rank_bound(reg, rank, 600, ids, qlb, qub),
                                                      orc.regression_rank_bound(reg, rank, 600, ids, qlb, qub)))
    for k in (1, 7, 25):
        a, _ = R.qs_retrieval(un, item, 9, rank, thr, query, k)
        b, _ = orc.qs_retrieval(un, item, 9, rank, thr, query, k)
        assert same_results(a, b)


@pytest.mark.skipif(not (Reference.available() and os.path.exists(REF_DATASET + "_user.fvecs")),
                    reason="reference dataset or oracle/_ref not present")
def test_oracle_matches_reference_on_bundled_dataset(orc):
    def fvecs(p):
        a = np.fromfile(p, dtype=np.int32)
        return a.reshape(-1, a[0] + 1)[:, 1:].view(np.float32).copy()

    R = Reference(n_thread=4)
    user = R.normalize(fvecs(REF_DATASET + "_user.fvecs"))
    item = fvecs(REF_DATASET + "_data_item.fvecs")
    query = fvecs(REF_DATASET + "_query_item.fvecs")
    si = R.sample_item(item.shape[0], 150)
    accu = R.query_rank_distribution(user, item, si)
    _, accu_o = orc.query_rank_distribution(user, item, si)
    assert np.array_equal(accu, accu_o)
    kth, sid = R.sort_kth_rank(accu, 40)
    rank, _ = R.find_optimal_sample_rank(user.shape[0], item.shape[0], 20, si, accu, 40)
    assert np.array_equal(rank, orc.optimal_sample_rank(user.shape[0], item.shape[0], 20, kth, accu[sid])[0])
    thr = R.build_thresholds(user, item, rank)
    ti, su, cd = R.svd_build(user, item)
    reg = R.fit_regression(thr, item.shape[0], rank)
    for k in (10, 20, 30):  # run_rkr.py:104
        a, _ = R.qs_retrieval(user, item, cd, rank, thr, query, k)
        b, _ = orc.qs_retrieval(user, item, cd, rank, thr, query, k)
        assert same_results(a, b)
        a, _ = R.qsrp_retrieval(user, su, ti, item, cd, rank, thr, rank, reg, query, k)
        b, _ = orc.qsrp_retrieval(user, su, ti, item, cd, rank, thr, rank, reg, query, k)
        assert same_results(a, b)
