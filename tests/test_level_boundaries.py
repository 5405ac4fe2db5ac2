"""The oracle's per-user level boundaries (orc_level_boundaries), the checker for level-boundary tables:
at every finite boundary B of level L the reference's rank bound (ComputeRankBound,
NormalLinearRegressionLP.hpp:326-380) has level <= L at B and > L one binary32 value below B, on both
sides (the lower bound as a function of qlb, the upper bound of qub), for fitted and capped users; the
boundaries do not rise with L; and a random score's level lies between the two boundaries around it."""
import numpy as np

from checkers import Oracle


def level(orc, rec, rank, n_item, q, side):
    lb, ub = orc.regression_rank_bound(rec[None, :], rank, n_item, [0], [q], [q])
    r = int(ub[0]) if side else int(lb[0])
    S = len(rank)
    return 0 if r == 0 else (S + 1 if r == n_item else int(np.searchsorted(rank, r)) + 1)


def test_level_boundaries_are_exact():
    orc = Oracle()
    rng = np.random.default_rng(3)
    n_item, S, stride = 17770, 512, 16
    rank = np.sort(rng.choice(np.arange(1, n_item - 1), S, replace=False)).astype(np.int32)
    thr = -np.sort(-(rng.standard_normal((5, S)) * rng.uniform(0.05, 0.4, (5, 1))).astype(np.float32), axis=1)
    reg = orc.fit_regression(thr)
    capped = reg[0].copy()
    capped[4] = np.float32(S)
    n_out = (S + 1) // stride + 2
    for rec in list(reg) + [capped]:
        for side in (0, 1):
            B = orc.level_boundaries(rec, rank, n_item, stride, side, n_out)
            assert np.all(B[1:] <= B[:-1])  # a looser level cap needs no higher score
            for g, b in enumerate(B):
                L = g * stride
                if np.isfinite(b):
                    assert level(orc, rec, rank, n_item, b, side) <= L
                    assert level(orc, rec, rank, n_item, np.nextafter(b, np.float32(-np.inf)), side) > L
            smin, smax = float(rec[6]), float(rec[5])
            for q in rng.uniform(smin - 0.05, smax + 0.05, 40).astype(np.float32):
                lv = level(orc, rec, rank, n_item, q, side)
                # the caps q reaches form a suffix g*, ..., n_out - 1: level <= g* stride, > (g* - 1) stride
                gs = len(B) - int(np.sum(B <= q))
                assert gs == len(B) or lv <= gs * stride
                assert gs == 0 or lv > (gs - 1) * stride
