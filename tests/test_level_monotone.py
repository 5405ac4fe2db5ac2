"""The reference's regression rank bound (NormalLinearRegressionLP::ComputeRankBound,
NormalLinearRegressionLP.hpp:326-380, through the oracle) never rises as the score grows, for either
side: over sampled scores across [smin, smax] and over runs of consecutive binary32 scores across level
boundaries.  A per-user table of the scores at level boundaries then gives a score's level exactly."""
import numpy as np

from checkers import Oracle
from test_level_screen import near_integer_scores


def bounds(orc, rec, rank, n_item, qs):
    L, H = [], []
    for q in qs:
        lb, ub = orc.regression_rank_bound(rec[None, :], rank, n_item, [0], [q], [q])
        L.append(int(lb[0]))
        H.append(int(ub[0]))
    return np.array(L), np.array(H)


def test_rank_bound_is_monotone_in_the_score():
    orc = Oracle()
    rng = np.random.default_rng(1)
    n_item, S = 17770, 512
    rank = np.sort(rng.choice(np.arange(1, n_item - 1), S, replace=False)).astype(np.int32)
    thr = -np.sort(-(rng.standard_normal((8, S)) * rng.uniform(0.05, 0.4, (8, 1))).astype(np.float32), axis=1)
    reg = orc.fit_regression(thr)
    for u in range(reg.shape[0]):
        smax, smin = float(reg[u, 5]), float(reg[u, 6])
        qs = np.sort(np.concatenate([np.linspace(smin - 0.05, smax + 0.05, 1500),
                                     rng.uniform(smin, smax, 500)]).astype(np.float32))
        L, H = bounds(orc, reg[u], rank, n_item, qs)
        assert not np.any(np.diff(L) > 0) and not np.any(np.diff(H) > 0)
        for q0 in near_integer_scores(orc, reg[u], S, 61)[::3]:
            run = [q0]
            for _ in range(24):
                run.insert(0, np.nextafter(run[0], np.float32(-np.inf)))
                run.append(np.nextafter(run[-1], np.float32(np.inf)))
            L, H = bounds(orc, reg[u], rank, n_item, run)
            assert not np.any(np.diff(L) > 0) and not np.any(np.diff(H) > 0)
