"""User sharding on the CPU: the count exchange, the merge of the shards' parts, and the sharded query
scheme against the reference's own outputs.

The scheme (include/rkr.h, "user shards"): every shard selects from per-query counts summed over the
shards, classifies, refines and assembles its own users, and the host merges the parts.  The oracle's
sharded restatement (oracle/rkr_oracle.c, orc_*_retrieval_shard) runs it here on the CPU with the
library's own exchange and merge (librkr_b200.so: rkr_host_exchange, rkr_shard_merge, host code only)
and with rkr_b200.shard.TorchExchange over two `gloo` ranks; the merged answers must equal the golden
vectors that the reference's own code wrote (tests/golden).  The engine's sharded GPU path is
checked against the same oracle in tests/test_gpu_shard.py.
"""
import os
import socket
import threading

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import rkr_b200 as rk
from checkers import Oracle
from rkr_b200.shard import TorchExchange, shard_users

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def bits(a):
    return np.ascontiguousarray(a).view(np.int32).reshape(-1)


def same(a, b):
    return np.array_equal(bits(a), bits(b))


# ---- the merge ---------------------------------------------------------------------------------------

def rec(u, r, s=0.5):
    return (u, r, s)


def test_merge_orders_results_by_shard_then_candidates_by_rank_and_user():
    ks = np.array([5, 3], np.int32)
    # query 0: shard 0 has results 2, 7 and candidates (rank 9, user 4), (rank 12, user 1); shard 1 has
    # result 30 and candidates (rank 9, user 31), (rank 10, user 40)
    p0 = np.array([rec(2, 1), rec(7, 1), rec(4, 9), rec(1, 12), rec(-1, -1),
                   rec(3, 2), rec(-1, -1), rec(-1, -1)], rk.USER_RANK)
    p1 = np.array([rec(30, 1), rec(31, 9), rec(40, 10), rec(-1, -1), rec(-1, -1),
                   rec(50, 4), rec(51, 4), rec(-1, -1)], rk.USER_RANK)
    f0, f1 = np.array([2, 0], np.int32), np.array([1, 0], np.int32)
    out = rk.shard_merge(ks, [p0, p1], [f0, f1])
    assert list(out["user_id"][:5]) == [2, 7, 30, 4, 31]
    assert list(out["rank"][:5]) == [1, 1, 1, 9, 9]
    # query 1: no results; candidates (2, 3), (4, 50), (4, 51) by (rank, user id)
    assert list(out["user_id"][5:]) == [3, 50, 51]


def test_merge_truncates_results_to_k_and_sums_stats():
    ks = np.array([2], np.int32)
    p0 = np.array([rec(0, 0), rec(1, 0)], rk.USER_RANK)
    p1 = np.array([rec(5, 0), rec(-1, -1)], rk.USER_RANK)
    st0 = np.zeros(1, rk.QUERY_STATS)
    st1 = np.zeros(1, rk.QUERY_STATS)
    st0[0] = (7, 3, 2, 4, 100, 1000)
    st1[0] = (7, 3, 1, 2, 50, 70)
    out, st = rk.shard_merge(ks, [p0, p1], [np.array([2], np.int32), np.array([1], np.int32)], [st0, st1])
    assert list(out["user_id"]) == [0, 1]
    assert tuple(st[0]) == (7, 3, 3, 6, 150, 1070)


def test_merge_rejects_bad_fronts():
    ks = np.array([2], np.int32)
    p = np.zeros(2, rk.USER_RANK)
    with pytest.raises(rk.RkrError):
        rk.shard_merge(ks, [p], [np.array([3], np.int32)])


# ---- the in-process exchange ------------------------------------------------------------------------------

def test_host_exchange_sums_over_threads():
    n = 3
    ex = rk.HostExchange(n, timeout_s=20.0)
    bufs = [np.arange(10, dtype=np.int32) * (i + 1) for i in range(n)]
    rcs = [None] * n

    def member(i):
        for step in range(4):  # repeated exchanges of different sizes reuse the group
            b = bufs[i][:10 - step]
            rcs[i] = ex.fn(ex.ctx, b.ctypes.data, b.shape[0], None)
            if rcs[i]:
                return

    ts = [threading.Thread(target=member, args=(i,)) for i in range(n)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert rcs == [0] * n
    # step 0 sums j, 2j, 3j to 6j on every member; each later step covering element j triples it
    for i in range(n):
        assert list(bufs[i]) == [6 * j * 3 ** min(3, 9 - j) for j in range(10)]
    ex.close()


def test_host_exchange_times_out_without_every_member():
    ex = rk.HostExchange(2, timeout_s=0.2)
    b = np.ones(4, np.int32)
    assert ex.fn(ex.ctx, b.ctypes.data, 4, None) != 0
    assert ex.fn(ex.ctx, b.ctypes.data, 4, None) != 0  # a broken group fails at once
    ex.close()


# ---- the scheme on the oracle ----------------------------------------------------------------------------

def run_shard(orc, g, method, k, start, end, exchange, qip_state=None):
    n_total = g["user_norm"].shape[0]
    sl = slice(start, end)
    if method == "QS":
        return orc.qs_retrieval_shard(g["user_norm"][sl], g["item"], int(g["check_dim"]), g["opt_rank"],
                                      g["thr"][sl], g["query"], k, start, n_total, exchange)
    if method == "US":
        q100 = np.concatenate([g["query"]] * (100 // g["query"].shape[0] + 1))[:100]
        return orc.us_retrieval_shard(g["user_norm"][sl], g["item"], g["uni_rank"], g["thr_uni"][sl], q100, k,
                                      start, n_total, exchange)
    return orc.qsrp_retrieval_shard(g["user_norm"][sl], g["svd_user"][sl], g["transfer_item"], g["item"],
                                    int(g["check_dim"]), g["opt_rank"], g["thr"][sl], g["opt_rank"], g["reg"][sl],
                                    g["query"], k, start, n_total, exchange, qip_state)


GOLDEN_KEY = {"QS": "qs", "QSRPNormalLP": "qsrp", "US": "us"}


@pytest.mark.parametrize("case", ["small", "fakenormal"])
@pytest.mark.parametrize("n_shards", [2, 3])
@pytest.mark.parametrize("method", ["QS", "QSRPNormalLP", "US"])
def test_sharded_oracle_threads_match_golden(case, n_shards, method):
    orc = Oracle()
    g = load(case)
    k = int(g["topk"])
    n_total = g["user_norm"].shape[0]
    ex = rk.HostExchange(n_shards, timeout_s=60.0)
    res = [None] * n_shards

    def member(s):
        start, end = shard_users(n_total, n_shards, s)
        res[s] = run_shard(orc, g, method, k, start, end, (ex.fn, ex.ctx))

    ts = [threading.Thread(target=member, args=(s,)) for s in range(n_shards)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert all(r is not None for r in res)
    nq = res[0][0].shape[0]
    ks = np.full(nq, k, np.int32)
    out, st = rk.shard_merge(ks, [r[0].reshape(-1) for r in res], [r[1] for r in res], [r[2] for r in res])
    want, wst = g[GOLDEN_KEY[method]], g[GOLDEN_KEY[method] + "_stats"]
    assert same(out, want[:nq])
    for f in ("n_prune", "n_result", "n_refine", "ip_cost"):
        assert np.array_equal(st[f], wst[f][:nq]), f
    ex.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = Oracle()
        ex = TorchExchange()
        for case in ("small", "fakenormal"):
            g = load(case)
            k = int(g["topk"])
            start, end = shard_users(g["user_norm"].shape[0], world, rank)
            for method in ("QS", "QSRPNormalLP", "US"):
                out, front, st = run_shard(orc, g, method, k, start, end, (ex.fn, None))
                got = [None] * world
                dist.all_gather_object(got, (out.reshape(-1), front, st))
                nq = out.shape[0]
                merged, mst = rk.shard_merge(np.full(nq, k, np.int32), [x[0] for x in got], [x[1] for x in got],
                                             [x[2] for x in got])
                np.savez(os.path.join(out_dir, f"r{rank}_{case}_{method}.npz"), out=merged, st=mst)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sharded_queries_match_golden(tmp_path):
    world = 2
    mp.spawn(_gloo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for case in ("small", "fakenormal"):
        g = load(case)
        for method in ("QS", "QSRPNormalLP", "US"):
            want, wst = g[GOLDEN_KEY[method]], g[GOLDEN_KEY[method] + "_stats"]
            for r in range(world):
                x = np.load(os.path.join(tmp_path, f"r{r}_{case}_{method}.npz"))
                nq = x["out"].shape[0] // int(g["topk"])
                assert same(x["out"], want[:nq]), (case, method, r)
                assert np.array_equal(x["st"]["ip_cost"], wst["ip_cost"][:nq])
                assert np.array_equal(x["st"]["n_refine"], wst["n_refine"][:nq])
