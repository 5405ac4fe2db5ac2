"""The serving loop (rkr_server_*): continuous batching over a resident index.

Requests -- each a set of query items with a top-k per item -- are submitted from several host
threads at once, so that the server batches requests of different sizes and k together, runs several
batches at a time on its workers' streams and replays the phase-1 graphs it captured.  Every
request's rows must equal what the same request gets alone from a freshly reset index (rkr_query),
bit for bit, and -- for a sample -- what the oracle gives for it alone; the result of a request must
not depend on the mix it was served in.
"""
import threading

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle

pytestmark = pytest.mark.gpu


def same(a, b):
    a = np.ascontiguousarray(a).view(np.int32).reshape(-1)
    b = np.ascontiguousarray(b).view(np.int32).reshape(-1)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.fixture(scope="module")
def served():
    orc = Oracle()
    rng = np.random.default_rng(404)
    n_user, n_item, d = 3000, 4000, 48
    user = orc.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, 40), np.linspace(40, n_item - 2, 60).astype(int)])).astype(np.int32)
    thr = orc.build_thresholds(user, item, rank)
    reg = orc.fit_regression(thr)
    ti, su, cd = R.svd_build(user, 0.7)
    ix = R.Index(user, item)
    ix.load_sample_search(rank, thr)
    ix.load_svd(cd, ti, su)
    ix.load_regression(rank, reg)
    reqs = []
    for i in range(60):
        n = int(rng.integers(1, 41))
        if i % 2:
            q = item[rng.choice(n_item, n, replace=False)].copy()
        else:
            q = (rng.standard_normal((n, d)) / np.sqrt(d)).astype(np.float32)
        reqs.append((q, rng.integers(1, 80, n).astype(np.int32)))
    yield dict(ix=ix, orc=orc, user=user, item=item, rank=rank, thr=thr, reg=reg, ti=ti, su=su, cd=cd, reqs=reqs)
    ix.close()


@pytest.mark.parametrize("method", ["QSRPNormalLP", "QS"])
def test_each_request_equals_its_result_alone(served, method):
    ix, reqs = served["ix"], served["reqs"]
    results = [None] * len(reqs)
    with R.Server(ix, method=method, max_batch_queries=256, n_workers=2) as srv:
        def client(idx):
            tickets = [(i, srv.submit(*reqs[i])) for i in idx]
            for i, t in tickets:
                results[i] = srv.wait(t, timeout=120.0)[0]
        threads = [threading.Thread(target=client, args=(list(range(j, len(reqs), 4)),)) for j in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        c = srv.counters()
    assert c["requests"] == len(reqs) and c["queries"] == sum(q.shape[0] for q, _ in reqs)
    assert c["batches"] < len(reqs)  # requests were batched together
    for i, (q, ks) in enumerate(reqs):
        ix.reset_state()
        alone = ix.query(method, q, ks)
        assert results[i] is not None and len(results[i]) == len(alone)
        for a, b in zip(results[i], alone):
            assert same(a, b), (method, i)


def test_requests_match_the_oracle_alone(served):
    """A few requests through the server against the oracle, each from a fresh state."""
    s = served
    orc = s["orc"]
    with R.Server(s["ix"], method="QSRPNormalLP", max_batch_queries=64, n_workers=2) as srv:
        tickets = [(i, srv.submit(*s["reqs"][i])) for i in range(0, 12)]
        got = {i: srv.wait(t, timeout=120.0)[0] for i, t in tickets}
        # the same requests again: graphs captured on the way are replayed, results unchanged
        tickets = [(i, srv.submit(*s["reqs"][i])) for i in range(0, 12)]
        again = {i: srv.wait(t, timeout=120.0)[0] for i, t in tickets}
    for i in range(0, 12, 3):
        q, ks = s["reqs"][i]
        state = np.zeros(s["user"].shape[0], np.float32)
        for j in range(q.shape[0]):
            want, _ = orc.qsrp_retrieval(s["user"], s["su"], s["ti"], s["item"], s["cd"], s["rank"], s["thr"],
                                         s["rank"], s["reg"], q[j:j + 1], int(ks[j]), qip_state=state)
            assert same(got[i][j], want[0]), (i, j)
    for i in got:
        for a, b in zip(got[i], again[i]):
            assert same(a, b)


def test_server_rejects_bad_requests(served):
    with R.Server(served["ix"], method="QS", max_batch_queries=16, n_workers=1) as srv:
        q, _ = served["reqs"][0]
        with pytest.raises(R.RkrError):
            srv.submit(np.concatenate([q] * 20)[:17], np.ones(17, np.int32))  # larger than a batch
        with pytest.raises(R.RkrError):
            srv.submit(q, np.zeros(q.shape[0], np.int32))  # k = 0
    with pytest.raises(R.RkrError):
        R.Server(served["ix"], method="US")
