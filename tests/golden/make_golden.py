"""Generates tests/golden/*.npz: seeded synthetic inputs plus the outputs of the reference's own
code for them (oracle/_ref/librkr_ref.so, built by `make -C oracle ref` from the reference
sources).  Run from the repository root:  python tests/golden/make_golden.py

Each case is one run of the reference pipeline on i.i.d. normal vectors:
  users L2-normalised -> sampled items (mt19937(0) shuffle) -> query-rank distribution ->
  k-th ranks -> optimal and uniform sample ranks -> thresholds -> SVD transform -> regression
  models -> QS / QSRPNormalLP / US retrieval.
The SVD transform and regression models are produced by the harness's stand-ins (oracle/ref_shim);
they are inputs to the query stage and are stored, so every consumer reads the same values.

refdataset.npz is the same pipeline on the reference's own bundled dataset
(dataset/fake-normal-30d: 1,000 users, 5,000 items, 100 queries, d = 30, read from the reference
checkout, $RKR_REFERENCE_ROOT or ../reference) with the parameters its driver script runs
(run_rkr.py:73-78,104: 150 sampled items, sample_topk 40, 20 sampled ranks, k in {10, 20, 30}); each
k is a separate run from a fresh index, as each rri call is.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from checkers import Reference, reference_root  # noqa: E402

CASES = {
    # name: (n_user, n_item, d, n_query, std, n_sample, n_sample_item, sample_topk, topk, seed)
    "small": (300, 800, 30, 30, 1.0, 16, 100, 20, 10, 11),
    "fakenormal": (400, 1000, 30, 40, 5.0, 20, 150, 40, 20, 12),
}


def make(name, n_user, n_item, d, n_query, std, n_sample, n_sample_item, sample_topk, topk, seed):
    rng = np.random.default_rng(seed)
    user = (rng.standard_normal((n_user, d)) * std).astype(np.float32)
    item = (rng.standard_normal((n_item, d)) * std).astype(np.float32)
    qid = rng.choice(n_item, size=n_query // 2, replace=False)
    query = np.concatenate([item[qid], (rng.standard_normal((n_query - n_query // 2, d)) * std).astype(np.float32)])
    R = Reference(n_thread=4)
    un = R.normalize(user)
    sample_item = R.sample_item(n_item, n_sample_item)
    accu = R.query_rank_distribution(un, item, sample_item)
    sort_kth, sort_sid = R.sort_kth_rank(accu, sample_topk)
    opt_rank, opt_cost = R.find_optimal_sample_rank(n_user, n_item, n_sample, sample_item, accu, sample_topk)
    uni_rank = R.uniform_sample_rank(n_item, n_sample)
    thr = R.build_thresholds(un, item, opt_rank)
    thr_uni = R.build_thresholds(un, item, uni_rank)
    transfer_item, svd_user, check_dim = R.svd_build(un, item)
    reg = R.fit_regression(thr, n_item, opt_rank)
    qs, qs_st = R.qs_retrieval(un, item, check_dim, opt_rank, thr, query, topk)
    qsrp, qsrp_st = R.qsrp_retrieval(un, svd_user, transfer_item, item, check_dim, opt_rank, thr, opt_rank, reg,
                                     query, topk)
    us, us_st = R.us_retrieval(un, item, uni_rank, thr_uni, np.concatenate([query] * (100 // n_query + 1))[:100],
                               topk)
    out = dict(user=user, item=item, query=query, user_norm=un, sample_item=sample_item, accu=accu,
               sort_kth=sort_kth, sort_sid=sort_sid, opt_rank=opt_rank, opt_cost=np.int64(opt_cost),
               uni_rank=uni_rank, thr=thr, thr_uni=thr_uni, transfer_item=transfer_item, svd_user=svd_user,
               check_dim=np.int32(check_dim), reg=reg, topk=np.int32(topk), sample_topk=np.int32(sample_topk),
               qs=qs, qs_stats=qs_st, qsrp=qsrp, qsrp_stats=qsrp_st, us=us, us_stats=us_st)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "check_dim", check_dim, "opt_rank", opt_rank, "refine/q", qs_st["n_refine"].mean())


def fvecs(path):
    a = np.fromfile(path, dtype=np.int32)
    return a.reshape(-1, a[0] + 1)[:, 1:].view(np.float32).copy()


def make_refdataset():
    base = os.path.join(reference_root(), "dataset", "fake-normal-30d", "fake-normal-30d")
    user = fvecs(base + "_user.fvecs")
    item = fvecs(base + "_data_item.fvecs")
    query = fvecs(base + "_query_item.fvecs")
    n_user, n_item = user.shape[0], item.shape[0]
    n_sample_item, sample_topk, n_sample, topks = 150, 40, 20, (10, 20, 30)
    R = Reference(n_thread=4)
    un = R.normalize(user)
    sample_item = R.sample_item(n_item, n_sample_item)
    accu = R.query_rank_distribution(un, item, sample_item)
    opt_rank, opt_cost = R.find_optimal_sample_rank(n_user, n_item, n_sample, sample_item, accu, sample_topk)
    uni_rank = R.uniform_sample_rank(n_item, n_sample)
    thr = R.build_thresholds(un, item, opt_rank)
    thr_uni = R.build_thresholds(un, item, uni_rank)
    transfer_item, svd_user, check_dim = R.svd_build(un, item)
    reg = R.fit_regression(thr, n_item, opt_rank)
    out = dict(user=user, item=item, query=query, user_norm=un, sample_item=sample_item, accu=accu,
               opt_rank=opt_rank, opt_cost=np.int64(opt_cost), uni_rank=uni_rank, thr=thr, thr_uni=thr_uni,
               transfer_item=transfer_item, svd_user=svd_user, check_dim=np.int32(check_dim), reg=reg,
               sample_topk=np.int32(sample_topk), topks=np.array(topks, np.int32))
    for k in topks:
        out[f"qs_{k}"], out[f"qs_stats_{k}"] = R.qs_retrieval(un, item, check_dim, opt_rank, thr, query, k)
        out[f"qsrp_{k}"], out[f"qsrp_stats_{k}"] = R.qsrp_retrieval(un, svd_user, transfer_item, item, check_dim,
                                                                    opt_rank, thr, opt_rank, reg, query, k)
        out[f"us_{k}"], out[f"us_stats_{k}"] = R.us_retrieval(un, item, uni_rank, thr_uni, query, k)
    np.savez_compressed(os.path.join(HERE, "refdataset.npz"), **out)
    print("refdataset check_dim", check_dim, "opt_rank", opt_rank)


if __name__ == "__main__":
    which = sys.argv[1:] or list(CASES) + ["refdataset"]
    for k in which:
        if k == "refdataset":
            make_refdataset()
        else:
            make(k, *CASES[k])
