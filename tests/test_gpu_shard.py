"""User shards on the GPU: indexes over disjoint user ranges, driven by host threads on one GPU and
exchanging their per-query counts through rkr_host_exchange (the shards' kernels never wait for one
another on the device: each exchange waits on the host between launches).  The merged answers must
equal the whole index's (rkr_query), the reference's golden outputs, and each shard's part the
oracle's sharded restatement, bit for bit, with every counter.
"""
import os
import threading
from datetime import timedelta

import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle
from rkr_b200.shard import shard_users

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STATS = ("n_prune", "n_result", "n_refine", "n_candidate", "n_compute_item", "ip_cost")


def load(case):
    return dict(np.load(os.path.join(GOLDEN, case + ".npz")))


def same(a, b):
    a = np.ascontiguousarray(a).view(np.int32).reshape(-1)
    b = np.ascontiguousarray(b).view(np.int32).reshape(-1)
    return a.shape == b.shape and np.array_equal(a, b)


def make_shards(user, item, bounds, sample_rank, thr, check_dim, reg=None, reg_rank=None, svd=None, timeout=60.0):
    """One index per user range, with its rows of the per-user arrays, made shards of one group."""
    n = len(bounds)
    ex = R.HostExchange(n, timeout_s=timeout)
    shards = []
    for s, (a, b) in enumerate(bounds):
        ix = R.Index(user[a:b], item)
        if check_dim is not None:
            ix.set_check_dim(check_dim)
        ix.load_sample_search(sample_rank, thr[a:b])
        if svd is not None:
            ti, su, cd = svd
            ix.load_svd(cd, ti, su[a:b])
        if reg is not None:
            ix.load_regression(reg_rank, reg[a:b])
        ix.set_shard(s, n, a, user.shape[0], ex)
        shards.append(ix)
    return shards, ex


def run_threads(shards, fn):
    """fn(shard index, index) on one host thread per shard; the results in shard order."""
    res, err = [None] * len(shards), [None] * len(shards)

    def member(s):
        try:
            res[s] = fn(s, shards[s])
        except Exception as e:  # noqa: BLE001 -- re-raised below
            err[s] = e

    ts = [threading.Thread(target=member, args=(s,)) for s in range(len(shards))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for e in err:
        if e is not None:
            raise e
    return res


def sharded_query(shards, method, query, ks):
    parts = run_threads(shards, lambda s, ix: ix.shard_query(method, query, ks, stats=True))
    n = parts[0][1].shape[0]
    out, st = R.shard_merge(ks[:n], [p[0] for p in parts], [p[1] for p in parts], [p[2] for p in parts])
    return out, st, parts


def close_all(shards, ex):
    for ix in shards:
        ix.close()
    ex.close()


@pytest.mark.parametrize("case", ["small", "fakenormal"])
@pytest.mark.parametrize("n_shards", [2, 3])
def test_shards_match_golden_and_oracle(case, n_shards):
    g = load(case)
    orc = Oracle()
    k = int(g["topk"])
    un, item, cd = g["user_norm"], g["item"], int(g["check_dim"])
    N = un.shape[0]
    bounds = [shard_users(N, n_shards, s) for s in range(n_shards)]
    svd = (g["transfer_item"], g["svd_user"], cd)
    shards, ex = make_shards(un, item, bounds, g["opt_rank"], g["thr"], cd, g["reg"], g["opt_rank"], svd)
    try:
        for method, key in (("QS", "qs"), ("QSRPNormalLP", "qsrp")):
            ks = np.full(g["query"].shape[0], k, np.int32)
            out, st, parts = sharded_query(shards, method, g["query"], ks)
            assert same(out, g[key]), method
            for f in ("n_prune", "n_result", "n_refine", "ip_cost"):
                assert np.array_equal(st[f], g[key + "_stats"][f]), (method, f)
            # each shard's part is the oracle's sharded restatement's (threads over the same exchange kind)
            oex = R.HostExchange(n_shards, timeout_s=60.0)

            def oracle_part(s, _ix):
                a, b = bounds[s]
                if method == "QS":
                    return orc.qs_retrieval_shard(un[a:b], item, cd, g["opt_rank"], g["thr"][a:b], g["query"], k, a, N,
                                                  (oex.fn, oex.ctx))
                return orc.qsrp_retrieval_shard(un[a:b], g["svd_user"][a:b], g["transfer_item"], item, cd,
                                                g["opt_rank"], g["thr"][a:b], g["opt_rank"], g["reg"][a:b],
                                                g["query"], k, a, N, (oex.fn, oex.ctx))
            want = run_threads(shards, oracle_part)
            oex.close()
            for s in range(n_shards):
                assert same(parts[s][0], want[s][0]), (method, s)
                assert np.array_equal(parts[s][1], want[s][1]), (method, s)
                for f in STATS:
                    assert np.array_equal(parts[s][2][f], want[s][2][f]), (method, s, f)
    finally:
        close_all(shards, ex)
    # US on its own sample ranks
    q100 = np.concatenate([g["query"]] * (100 // g["query"].shape[0] + 1))[:100]
    shards, ex = make_shards(un, item, bounds, g["uni_rank"], g["thr_uni"], None)
    try:
        out, st, _ = sharded_query(shards, "US", q100, np.full(100, k, np.int32))
        assert same(out, g["us"])
        assert np.array_equal(st["ip_cost"], g["us_stats"]["ip_cost"])
    finally:
        close_all(shards, ex)


@pytest.fixture(scope="module")
def scale():
    """A larger index (the tensor-core pair scores, the capped round-2 histogram, both compaction
    forms): 24,001 users x 6,000 items, d = 64, engine-built thresholds."""
    rng = np.random.default_rng(77)
    n_user, n_item, d = 24001, 6000, 64
    user = R.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, 30), np.linspace(30, n_item - 2, 98).astype(int)])).astype(np.int32)
    si = R.sample_item(n_item, 150)
    whole = R.Index(user, item)
    accu = whole.query_rank_distribution(si)
    thr = whole.build_sample_search(rank)
    reg = R.fit_regression(thr)
    ti, su, cd = R.svd_build(user, 0.7)
    whole.load_svd(cd, ti, su)
    whole.load_regression(rank, reg)
    nq = 300
    query = np.concatenate([item[rng.choice(n_item, nq // 2, replace=False)],
                            (rng.standard_normal((nq - nq // 2, d)) / np.sqrt(d)).astype(np.float32)])
    ks = rng.integers(1, 151, nq).astype(np.int32)
    yield dict(whole=whole, user=user, item=item, rank=rank, thr=thr, reg=reg, svd=(ti, su, cd), accu=accu, si=si,
               query=query, ks=ks)
    whole.close()


@pytest.mark.parametrize("split", [(0.29,), (0.5, 0.75)])
def test_shards_at_scale_match_the_whole_index(scale, split):
    S = scale
    N = S["user"].shape[0]
    cuts = [0] + [int(N * f) for f in split] + [N]
    bounds = list(zip(cuts[:-1], cuts[1:]))
    shards, ex = make_shards(S["user"], S["item"], bounds, S["rank"], S["thr"], S["svd"][2], S["reg"], S["rank"],
                             S["svd"])
    try:
        # the build's one exchange: every shard's query-rank counts
        accs = run_threads(shards, lambda s, ix: ix.query_rank_distribution(S["si"]))
        for a in accs:
            assert np.array_equal(a, S["accu"])
        for method in ("QS", "QSRPNormalLP"):
            S["whole"].reset_state()
            for ix in shards:
                ix.reset_state()
            # two batches: QSRPNormalLP's carried scores advance alike on the shards
            for b in range(2):
                q = S["query"][b::2]
                ks = S["ks"][b::2]
                want, wst = S["whole"].query(method, q, ks, stats=True)
                out, st, _ = sharded_query(shards, method, q, ks)
                assert same(out, np.concatenate(want)), (method, b)
                for f in STATS:
                    assert np.array_equal(st[f], wst[f]), (method, b, f)
    finally:
        close_all(shards, ex)


def test_shard_calls_are_checked(scale):
    S = scale
    N = S["user"].shape[0]
    shards, ex = make_shards(S["user"], S["item"], [(0, N // 2), (N // 2, N)], S["rank"], S["thr"], S["svd"][2])
    try:
        with pytest.raises(R.RkrError):
            shards[0].query("QS", S["query"][:2], S["ks"][:2])       # a shard answers shard_query only
        with pytest.raises(R.RkrError):
            R.Server(shards[0], method="QS")
        with pytest.raises(R.RkrError):
            S["whole"].shard_query("QS", S["query"][:2], S["ks"][:2])  # a whole index is not a shard
        with pytest.raises(R.RkrError):
            shards[0].set_shard(0, 2, N - shards[0].n_user + 1, N, ex)  # users beyond n_user_total
    finally:
        close_all(shards, ex)


def test_a_missing_shard_fails_the_query_instead_of_waiting(scale):
    """A shard whose partner never calls: the exchange's timeout fails the query on the host, and
    the index answers again once it is whole."""
    S = scale
    N = S["user"].shape[0]
    ix = R.Index(S["user"][:N // 2], S["item"])
    ix.set_check_dim(S["svd"][2])
    ix.load_sample_search(S["rank"], S["thr"][:N // 2])
    ex = R.HostExchange(2, timeout_s=1.0)
    try:
        ix.set_shard(0, 2, 0, N, ex)
        with pytest.raises(R.RkrError):
            ix.shard_query("QS", S["query"][:4], S["ks"][:4])
        ix.set_shard(0, 1, 0, N // 2, None)
        out = ix.query("QS", S["query"][:4], np.minimum(S["ks"][:4], 50))
        assert len(out) == 4
    finally:
        ix.close()
        ex.close()


def test_torch_exchange_on_the_engine_stream(scale):
    """rkr_b200.shard.TorchExchange with device counts (NCCL, one rank): a single-shard index that
    exchanges every count through torch.distributed answers as the whole index."""
    import torch
    import torch.distributed as dist
    from rkr_b200.shard import TorchExchange

    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True, timeout=timedelta(seconds=60))
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=timedelta(seconds=60))
    S = scale
    N = S["user"].shape[0]
    ix = R.Index(S["user"], S["item"])
    try:
        ti, su, cd = S["svd"]
        ix.set_check_dim(cd)
        ix.load_sample_search(S["rank"], S["thr"])
        ix.load_svd(cd, ti, su)
        ix.load_regression(S["rank"], S["reg"])
        tex = TorchExchange(None, torch.device("cuda", 0))
        ix.set_shard(0, 1, 0, N, (tex.fn, None))
        S["whole"].reset_state()
        q, ks = S["query"][:64], S["ks"][:64]
        for method in ("QS", "QSRPNormalLP"):
            part, front, st = ix.shard_query(method, q, ks, stats=True)
            out, mst = R.shard_merge(ks, [part], [front], [st])
            want, wst = S["whole"].query(method, q, ks, stats=True)
            assert same(out, np.concatenate(want)), method
            for f in STATS:
                assert np.array_equal(mst[f], wst[f]), (method, f)
    finally:
        ix.close()
        dist.destroy_process_group()
