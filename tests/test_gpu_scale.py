"""GPU parity at full size: 480,189 users x 17,770 items, d = 150, 512 sampled thresholds per user.

The index is built on the device (query-rank distribution, OptimalPart ranks, thresholds) and on the
host (regression fit, SVD), with seeded synthetic data of the shape and value distribution the
throughput benchmark uses.  QSRPNormalLP retrieval through the C ABI must then equal the oracle bit
for bit -- user ids, ranks, scores and every per-query counter -- on queries drawn from the items and
from the same distribution, and, where oracle/_ref was built, the reference's own Retrieval.  The
full-size build is checked against the reference's own build stages on a subset of the users.
"""
import os

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle, Reference, ReferenceQsrp

pytestmark = pytest.mark.gpu

N_USER, N_ITEM, DIM, N_SAMPLE, N_SAMPLE_ITEM, SAMPLE_TOPK = 480189, 17770, 150, 512, 150, 100
STAT_FIELDS = ("n_prune", "n_result", "n_refine", "n_candidate", "n_compute_item", "ip_cost")


def same(a, b):
    a = np.ascontiguousarray(a).view(np.int32).reshape(-1)
    b = np.ascontiguousarray(b).view(np.int32).reshape(-1)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.fixture(scope="module")
def full():
    rng = np.random.default_rng(0)
    user = rng.standard_normal((N_USER, DIM), dtype=np.float32) * np.float32(1 / np.sqrt(DIM))
    item = rng.standard_normal((N_ITEM, DIM), dtype=np.float32) * np.float32(1 / np.sqrt(DIM))
    item *= np.exp(rng.normal(0.0, 0.3, (N_ITEM, 1))).astype(np.float32)
    un = R.normalize(user)
    ix = R.Index(un, item)
    si = R.sample_item(N_ITEM, N_SAMPLE_ITEM)
    accu = ix.query_rank_distribution(si)
    kth, sid = R.sort_kth_rank(accu, SAMPLE_TOPK)
    rank, _ = R.find_optimal_sample_rank(N_USER, N_ITEM, N_SAMPLE, kth, accu[sid])
    thr = ix.build_sample_search(rank)
    reg = R.fit_regression(thr)
    ti, su, cd = R.svd_build(un, 0.7)
    ix.load_svd(cd, ti, su)
    ix.load_regression(rank, reg)
    qrng = np.random.default_rng(77)
    query = np.concatenate([item[qrng.choice(N_ITEM, 10, replace=False)],
                            (qrng.standard_normal((6, DIM)) / np.sqrt(DIM)).astype(np.float32)])
    yield dict(ix=ix, un=un, item=item, rank=rank, thr=thr, reg=reg, ti=ti, su=su, cd=cd, query=query)
    ix.close()


@pytest.mark.parametrize("topk", [100, 50, 10])
def test_qsrp_full_size_matches_oracle(full, topk):
    orc = Oracle()
    ix = full["ix"]
    ix.reset_state()
    state = np.zeros(N_USER, np.float32)
    a, sa = ix.retrieval("QSRPNormalLP", full["query"], topk, stats=True)
    b, sb = orc.qsrp_retrieval(full["un"], full["su"], full["ti"], full["item"], full["cd"], full["rank"], full["thr"],
                               full["rank"], full["reg"], full["query"], topk, qip_state=state)
    for f in STAT_FIELDS:
        assert np.array_equal(sa[f], sb[f]), (f, sa[f], sb[f])
    assert same(a, b)


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_qsrp_full_size_matches_reference(full):
    import os
    ref = ReferenceQsrp(full["un"], full["su"], full["ti"], full["item"], full["cd"], full["rank"], full["thr"],
                        full["rank"], full["reg"], os.cpu_count() or 1)
    try:
        b, sb, _ = ref.run(full["query"], 100)
    finally:
        ref.close()
    ix = full["ix"]
    ix.reset_state()
    a, sa = ix.retrieval("QSRPNormalLP", full["query"], 100, stats=True)
    for f in ("n_prune", "n_result", "n_refine", "ip_cost"):
        assert np.array_equal(sa[f], sb[f]), (f, sa[f], sb[f])
    assert same(a, b)


def test_qsrp_full_batch_matches_oracle_on_sample(full):
    """A 1,000-query batch (the throughput benchmark's batch) at full size: every 40th query's
    result ids, ranks and counters equal the oracle's.  Ids, ranks and counters do not depend on the
    scores carried between queries, so the sampled queries can be checked on their own."""
    orc = Oracle()
    ix = full["ix"]
    rng = np.random.default_rng(5)
    batch = full["item"][rng.choice(N_ITEM, 1000, replace=False)].copy()
    ix.reset_state()
    a, sa = ix.retrieval("QSRPNormalLP", batch, 100, stats=True)
    pick = np.arange(0, 1000, 40)
    b, sb = orc.qsrp_retrieval(full["un"], full["su"], full["ti"], full["item"], full["cd"], full["rank"], full["thr"],
                               full["rank"], full["reg"], batch[pick], 100)
    for f in STAT_FIELDS:
        assert np.array_equal(sa[f][pick], sb[f]), (f, sa[f][pick], sb[f])
    assert np.array_equal(a["user_id"][pick], b["user_id"])
    assert np.array_equal(a["rank"][pick], b["rank"])


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_full_size_build_matches_reference_on_user_subset(full):
    """The config-2 thresholds (built for all 480,189 users in the device's batched pipeline) of 2,000
    users spread over the whole range, and the query-rank distribution of those users over all 17,770
    items, equal the reference's own build stages (CPUScoreTable rows, sort, SampleSearch gather;
    QueryRankByComputation) bit for bit."""
    sub = np.linspace(0, N_USER - 1, 2000).astype(np.int64)
    ref = Reference(os.cpu_count() or 1)
    users = np.ascontiguousarray(full["un"][sub])
    t_ref = ref.build_thresholds(users, full["item"], full["rank"])
    assert same(full["thr"][sub], t_ref)
    si = R.sample_item(N_ITEM, N_SAMPLE_ITEM)
    with R.Index(users, full["item"]) as ix2:
        accu = ix2.query_rank_distribution(si)
    assert np.array_equal(accu, ref.query_rank_distribution(users, full["item"], si))
