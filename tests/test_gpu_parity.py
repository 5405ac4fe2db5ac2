"""GPU parity: every result of librkr_b200.so (through its C ABI) equals the reference's, bit for bit.

Expected values come from the committed golden fixtures (outputs of the reference's own code,
tests/golden/make_golden.py) and from the oracle (oracle/rkr_oracle.c) on fresh seeded inputs.
Comparisons are exact: user ids, ranks and the binary32 patterns of the reported scores.
"""
import os

import numpy as np
import pytest

import rkr_b200
from checkers import Oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(case):
    return dict(np.load(os.path.join(GOLDEN, case + ".npz")))


def same(a, b):
    a = np.ascontiguousarray(a).view(np.int32).reshape(-1)
    b = np.ascontiguousarray(b).view(np.int32).reshape(-1)
    return a.shape == b.shape and np.array_equal(a, b)


def first_diff(a, b):
    for q in range(a.shape[0]):
        if not same(a[q], b[q]):
            return q, a[q], b[q]
    return None


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def make_index(g):
    ix = rkr_b200.Index(g["user_norm"], g["item"])
    ix.set_check_dim(int(g["check_dim"]))
    ix.load_sample_search(g["opt_rank"], g["thr"])
    return ix


@pytest.mark.parametrize("case", ["small", "fakenormal"])
def test_qs_matches_golden(case):
    g = load(case)
    with make_index(g) as ix:
        out, st = ix.retrieval("QS", g["query"], int(g["topk"]), stats=True)
    assert same(out, g["qs"]), first_diff(out, g["qs"])
    assert np.array_equal(st["n_refine"], g["qs_stats"]["n_refine"])
    assert np.array_equal(st["n_prune"], g["qs_stats"]["n_prune"])
    assert np.array_equal(st["n_result"], g["qs_stats"]["n_result"])
    assert np.array_equal(st["ip_cost"], g["qs_stats"]["ip_cost"])


@pytest.mark.parametrize("case", ["small", "fakenormal"])
def test_qsrp_matches_golden(case):
    g = load(case)
    with make_index(g) as ix:
        ix.load_svd(int(g["check_dim"]), g["transfer_item"], g["svd_user"])
        ix.load_regression(g["opt_rank"], g["reg"])
        out, st = ix.retrieval("QSRPNormalLP", g["query"], int(g["topk"]), stats=True)
    assert same(out, g["qsrp"]), first_diff(out, g["qsrp"])
    assert np.array_equal(st["n_result"], g["qsrp_stats"]["n_result"])
    assert np.array_equal(st["n_prune"], g["qsrp_stats"]["n_prune"])
    assert np.array_equal(st["ip_cost"], g["qsrp_stats"]["ip_cost"])


@pytest.mark.parametrize("case", ["small", "fakenormal"])
def test_us_matches_golden(case):
    g = load(case)
    q100 = np.concatenate([g["query"]] * (100 // g["query"].shape[0] + 1))[:100]
    with rkr_b200.Index(g["user_norm"], g["item"]) as ix:
        ix.load_sample_search(g["uni_rank"], g["thr_uni"])
        out, st = ix.retrieval("US", q100, int(g["topk"]), stats=True)
    assert same(out, g["us"]), first_diff(out, g["us"])
    assert np.array_equal(st["ip_cost"], g["us_stats"]["ip_cost"])
    assert np.array_equal(st["n_refine"], g["us_stats"]["n_refine"])


@pytest.mark.parametrize("case", ["small", "fakenormal"])
def test_build_matches_golden(case, orc):
    g = load(case)
    with rkr_b200.Index(g["user_norm"], g["item"]) as ix:
        thr = ix.build_sample_search(g["opt_rank"])
        assert same(thr, g["thr"])
        accu = ix.query_rank_distribution(g["sample_item"])
        assert np.array_equal(accu, g["accu"])
        rows = ix.score_sort_batch(3, 17)
        assert same(rows, orc.score_sort_rows(g["user_norm"], g["item"], 3, 17))


def random_case(seed, n_user, n_item, d, n_query, std=1.0, in_set=0.5):
    rng = np.random.default_rng(seed)
    user = (rng.standard_normal((n_user, d)) * std).astype(np.float32)
    item = (rng.standard_normal((n_item, d)) * std * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    n_in = int(n_query * in_set)
    query = np.concatenate([item[rng.choice(n_item, n_in, replace=False)],
                            (rng.standard_normal((n_query - n_in, d)) * std).astype(np.float32)])
    return user, item, query


@pytest.mark.parametrize("shape,refine,scores,compact", [
    ((1001, 777, 30, 70), "tc", "tc", "sparse"), ((2500, 3000, 48, 130), "tc", "tc", "sparse"),
    ((640, 5000, 150, 64), "tc", "tc", "sparse"), ((1001, 777, 30, 70), "tiles", "tiles", "sparse"),
    ((640, 5000, 150, 64), "tiles", "tiles", "sparse"), ((2500, 3000, 48, 130), "tc", "tiles", "sparse"),
    ((1001, 777, 30, 70), "tc", "tc", "two_pass"), ((640, 5000, 150, 64), "tc", "tc", "two_pass")])
def test_random_qs_qsrp_us_match_oracle(shape, refine, scores, compact, orc, monkeypatch):
    """Both paths of the pair scores and of the refinement: tensor-core scores with exact
    resolution of undecided pairs ("tc") and the exact SIMT tiles ("tiles"); and both forms of the
    ordered compaction (sparse per-query lists, or the two-pass form for every query)."""
    monkeypatch.setenv("RKR_REFINE_TC", "1" if refine == "tc" else "0")
    monkeypatch.setenv("RKR_SCORES_TC", "1" if scores == "tc" else "0")
    monkeypatch.setenv("RKR_COMPACT_SPARSE", "1" if compact == "sparse" else "0")
    n_user, n_item, d, nq = shape
    user, item, query = random_case(sum(shape), n_user, n_item, d, nq)
    un = orc.normalize(user)
    rank = np.unique(np.concatenate([np.arange(0, 40), np.linspace(40, n_item - 1, 60).astype(int)])).astype(np.int32)
    rank = rank[rank < n_item - 1][:96]
    thr = orc.build_thresholds(un, item, rank)
    reg = orc.fit_regression(thr)
    import rkr_b200 as R
    ti, su, cd = R.svd_build(un, 0.7)
    with R.Index(un, item) as ix:
        t2 = ix.build_sample_search(rank)
        assert same(t2, thr)
        ix.load_svd(cd, ti, su)
        ix.load_regression(rank, reg)
        state = np.zeros(n_user, np.float32)
        for k in (1, 10, 57):
            a, sa = ix.retrieval("QS", query, k, stats=True)
            b, sb = orc.qs_retrieval(un, item, cd, rank, thr, query, k)
            assert same(a, b), ("QS", k, first_diff(a, b))
            for f in ("n_prune", "n_result", "n_refine", "ip_cost", "n_compute_item"):
                assert np.array_equal(sa[f], sb[f]), ("QS", k, f)
            a, sa = ix.retrieval("QSRPNormalLP", query, k, stats=True)
            b, sb = orc.qsrp_retrieval(un, su, ti, item, cd, rank, thr, rank, reg, query, k, qip_state=state)
            assert same(a, b), ("QSRP", k, first_diff(a, b))
            for f in ("n_prune", "n_result", "n_refine", "ip_cost", "n_compute_item"):
                assert np.array_equal(sa[f], sb[f]), ("QSRP", k, f)
        q100 = np.concatenate([query] * 2)[:100]
        a = ix.retrieval("US", q100, 10)
        b, _ = orc.us_retrieval(un, item, rank, thr, q100, 10)
        assert same(a, b)


def test_qsrp_state_carries_across_calls(orc):
    """Users accepted by the regression bound report the score held from earlier queries, across
    separate retrieval calls on the same index (QSRPNormalLP.hpp:73,109,213-218)."""
    g = load("fakenormal")
    k = int(g["topk"])
    with make_index(g) as ix:
        ix.load_svd(int(g["check_dim"]), g["transfer_item"], g["svd_user"])
        ix.load_regression(g["opt_rank"], g["reg"])
        state = np.zeros(g["user"].shape[0], np.float32)
        for part in (g["query"][:7], g["query"][7:19], g["query"][19:]):
            a = ix.retrieval("QSRPNormalLP", part, k)
            b, _ = orc.qsrp_retrieval(g["user_norm"], g["svd_user"], g["transfer_item"], g["item"],
                                      int(g["check_dim"]), g["opt_rank"], g["thr"], g["opt_rank"], g["reg"], part, k,
                                      qip_state=state)
            assert same(a, b), first_diff(a, b)
        ix.reset_state()
        a = ix.retrieval("QSRPNormalLP", g["query"], k)
    assert same(a, g["qsrp"])


def test_edge_cases(orc):
    g = load("small")
    with make_index(g) as ix:
        n_user = g["user"].shape[0]
        with pytest.raises(rkr_b200.RkrError):
            ix.retrieval("QS", g["query"], n_user + 1)
        with pytest.raises(rkr_b200.RkrError):
            ix.retrieval("QS", g["query"], 0)
        with pytest.raises(rkr_b200.RkrError):
            ix.retrieval("QSRPNormalLP", g["query"], 5)  # no regression / svd loaded
        assert ix.retrieval("QS", g["query"][:0], 5).shape[0] == 0
        full = ix.retrieval("QS", g["query"][:3], n_user)
        ref, _ = orc.qs_retrieval(g["user_norm"], g["item"], int(g["check_dim"]), g["opt_rank"], g["thr"],
                                  g["query"][:3], n_user)
        assert same(full, ref)
        one = ix.retrieval("QS", g["query"][:1], 1)
        ref, _ = orc.qs_retrieval(g["user_norm"], g["item"], int(g["check_dim"]), g["opt_rank"], g["thr"],
                                  g["query"][:1], 1)
        assert same(one, ref)


@pytest.mark.parametrize("compact", ["sparse", "two_pass"])
def test_mixed_k_batch_equals_one_call_per_query(orc, compact, monkeypatch):
    """rkr_query with a top-k per query: every query's entries equal the oracle's for that query
    alone with its k, called in order on the same index, so that QSRPNormalLP's carried scores
    advance exactly as across the reference's consecutive Retrieval calls."""
    monkeypatch.setenv("RKR_COMPACT_SPARSE", "1" if compact == "sparse" else "0")
    user, item, query = random_case(97, 1500, 2200, 48, 80)
    un = orc.normalize(user)
    rank = np.unique(np.concatenate([np.arange(0, 30), np.linspace(30, 2100, 50).astype(int)])).astype(np.int32)
    thr = orc.build_thresholds(un, item, rank)
    reg = orc.fit_regression(thr)
    ti, su, cd = rkr_b200.svd_build(un, 0.7)
    ks = np.random.default_rng(3).integers(1, 120, query.shape[0]).astype(np.int32)
    ks[:3] = (1, 1500, 4)
    with rkr_b200.Index(un, item) as ix:
        ix.load_sample_search(rank, thr)
        ix.load_svd(cd, ti, su)
        ix.load_regression(rank, reg)
        for method in ("QS", "QSRPNormalLP"):
            ix.reset_state()
            rows, st = ix.query(method, query, ks, stats=True)
            assert len(rows) == query.shape[0]
            state = np.zeros(un.shape[0], np.float32)
            for i, k in enumerate(ks):
                if method == "QS":
                    want, ws = orc.qs_retrieval(un, item, cd, rank, thr, query[i:i + 1], int(k))
                else:
                    want, ws = orc.qsrp_retrieval(un, su, ti, item, cd, rank, thr, rank, reg, query[i:i + 1], int(k),
                                                  qip_state=state)
                assert same(rows[i], want[0]), (method, i, int(k))
                for f in ("n_prune", "n_result", "n_refine", "ip_cost"):
                    assert st[f][i] == ws[f][0], (method, i, f)
        # US answers the first 100 queries per call
        q100 = np.concatenate([query, query])[:100]
        k100 = np.concatenate([ks, ks])[:100]
        with rkr_b200.Index(un, item) as ix2:
            ix2.load_sample_search(rank, thr)
            rows = ix2.query("US", q100, k100)
            assert len(rows) == 100
            for k in (int(k100[0]), int(k100[7])):
                want, _ = orc.us_retrieval(un, item, rank, thr, q100, k)
                for i in range(100):
                    if int(k100[i]) == k:
                        assert same(rows[i], want[i])
