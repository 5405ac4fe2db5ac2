"""GPU parity at the largest configuration: 1,000,990 users x 624,961 items, d = 150, 512 sampled
thresholds per user.  Score rows this long take the build's global-memory selection path (rows longer
than shared memory), and the refinement walks 625 K items per candidate.

The index is built on the device end to end (query-rank distribution, OptimalPart ranks, thresholds,
regression fit, SVD) from seeded synthetic data with the throughput benchmark's shapes and value
distributions.  QSRPNormalLP through the C ABI must equal the oracle bit for bit -- user ids, ranks,
scores and every per-query counter -- on queries drawn from the items and out of set, and the
thresholds and query-rank distribution of a subset of the users must equal the reference's own build
stages (where oracle/_ref was built).
"""
import os

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle, Reference

pytestmark = pytest.mark.gpu

N_USER, N_ITEM, DIM, N_SAMPLE, N_SAMPLE_ITEM, SAMPLE_TOPK = 1000990, 624961, 150, 512, 150, 100
STAT_FIELDS = ("n_prune", "n_result", "n_refine", "n_candidate", "n_compute_item", "ip_cost")


def same(a, b):
    a = np.ascontiguousarray(a).view(np.int32).reshape(-1)
    b = np.ascontiguousarray(b).view(np.int32).reshape(-1)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.fixture(scope="module")
def c4():
    rng = np.random.default_rng(4)
    user = rng.standard_normal((N_USER, DIM), dtype=np.float32) * np.float32(1 / np.sqrt(DIM))
    item = rng.standard_normal((N_ITEM, DIM), dtype=np.float32) * np.float32(1 / np.sqrt(DIM))
    item *= np.exp(rng.normal(0.0, 0.3, (N_ITEM, 1))).astype(np.float32)
    un = R.normalize(user)
    del user
    ix = R.Index(un, item)
    si = R.sample_item(N_ITEM, N_SAMPLE_ITEM)
    accu = ix.query_rank_distribution(si)
    kth, sid = R.sort_kth_rank(accu, SAMPLE_TOPK)
    rank, _ = R.find_optimal_sample_rank(N_USER, N_ITEM, N_SAMPLE, kth, accu[sid])
    del accu
    thr = ix.build_sample_search(rank)
    reg = ix.fit_regression()
    ti, su, cd = ix.svd_build(0.7)
    qrng = np.random.default_rng(44)
    query = np.concatenate([item[qrng.choice(N_ITEM, 3, replace=False)],
                            (qrng.standard_normal((2, DIM)) / np.sqrt(DIM)).astype(np.float32)])
    yield dict(ix=ix, un=un, item=item, rank=rank, thr=thr, reg=reg, ti=ti, su=su, cd=cd, query=query)
    ix.close()


def test_qsrp_config4_matches_oracle(c4):
    orc = Oracle()
    ix = c4["ix"]
    ix.reset_state()
    state = np.zeros(N_USER, np.float32)
    a, sa = ix.retrieval("QSRPNormalLP", c4["query"], 100, stats=True)
    b, sb = orc.qsrp_retrieval(c4["un"], c4["su"], c4["ti"], c4["item"], c4["cd"], c4["rank"], c4["thr"],
                               c4["rank"], c4["reg"], c4["query"], 100, qip_state=state)
    for f in STAT_FIELDS:
        assert np.array_equal(sa[f], sb[f]), (f, sa[f], sb[f])
    assert same(a, b)


def test_config4_device_fit_matches_host_fit(c4):
    """The regression records the device fitted for all 1,000,990 users equal the host fit's on a
    spread of users (the host fit is checked against the reference's golden records elsewhere)."""
    sub = np.linspace(0, N_USER - 1, 5000).astype(np.int64)
    assert same(c4["reg"][sub], R.fit_regression(c4["thr"][sub]))


@pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built (needs the reference sources)")
def test_config4_build_matches_reference_on_user_subset(c4):
    """Thresholds of 120 users spread over the whole range (built in the device's batched long-row
    pipeline for all users) and the query-rank distribution of those users over all 624,961 items
    equal the reference's own build stages bit for bit."""
    sub = np.linspace(0, N_USER - 1, 120).astype(np.int64)
    ref = Reference(os.cpu_count() or 1)
    users = np.ascontiguousarray(c4["un"][sub])
    assert same(c4["thr"][sub], ref.build_thresholds(users, c4["item"], c4["rank"]))
    si = R.sample_item(N_ITEM, N_SAMPLE_ITEM)
    with R.Index(users, c4["item"]) as ix2:
        accu = ix2.query_rank_distribution(si)
    assert np.array_equal(accu, ref.query_rank_distribution(users, c4["item"], si))
