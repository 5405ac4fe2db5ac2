"""The per-user level-boundary tables of the regression rank bound, restated on the CPU.

The device builds, per user and side, the smallest binary32 score T_g whose level (the reference's
ComputeRankBound, NormalLinearRegressionLP.hpp:326-380, lower bound of qlb / upper bound of qub) is
<= L_g (L_0 = 0, 14 steps to S, L_15 = S + 1), and a guard band around it
(reverse-k-ranks_b200/csrc/rkr_levels.cu); a score's coarse level (the smallest g with level <= L_g)
is then decided from the table wherever the score stays outside the bands.  Here:

* the band's premise: the reference's binary32 model value a CDFPhi((q - mu) / sigma) + b +- err
  differs from the same formula evaluated without roundings by less than a third of the margin the
  tables use;
* a restatement of the tables (boundaries from the oracle's orc_level_boundaries, bands from the
  model's double-precision crossing zone, as the kernel computes them) decides the coarse level of
  every probed score -- dense around each boundary, at its binary32 neighbours, and at random --
  exactly as the oracle's own levels give it, on fitted, steep, capped and extreme-score users;
* the screen decides no score inside a guard band, and decides scores just outside isolated ones.
"""
import math

import numpy as np
import pytest

from checkers import Oracle

E = 16  # table entries per side


def table_levels(S):
    """L_g: 0, then ceil(g S / 14) up to S, then S + 1 (lvt_level)."""
    return np.array([(g * S + E - 3) // (E - 2) for g in range(E - 1)] + [S + 1], np.int32)


def coarse(lv, S):
    """The smallest g with lv <= L_g (lvt_coarse)."""
    return int(np.searchsorted(table_levels(S), lv, side="left"))


A1, A2, A3, A4, A5, P = (float(np.float32(v)) for v in (0.254829592, -0.284496736, 1.421413741, -1.453152027,
                                                       1.061405429, 0.3275911))
SQRT2 = float(np.float32(math.sqrt(2.0)))


def model_value(rec, upper, q):
    """a Phi(z) + b +- err without the reference's binary32 roundings (double)."""
    a, b, mu, sigma, err = (float(x) for x in rec[:5])
    z = (q - mu) / sigma
    x = abs(z) / SQRT2
    t = 1.0 / (1.0 + P * x)
    y = 1.0 - (((((A5 * t + A4) * t) + A3) * t + A2) * t + A1) * t * math.exp(-x * x)
    phi = 0.5 * (1.0 + (-y if z < 0 else y))
    return a * phi + b + (-err if upper else err)


def model_margin(rec):
    a, b, err = (abs(float(x)) for x in (rec[0], rec[1], rec[4]))
    return a * 1.5e-6 + (a + b + err) * 6e-7 + 1e-6


def level(orc, rec, rank, n_item, q, side):
    lb, ub = orc.regression_rank_bound(rec[None, :], rank, n_item, [0], [q], [q])
    r = int(ub[0]) if side else int(lb[0])
    S = len(rank)
    return 0 if r == 0 else (S + 1 if r == n_item else int(np.searchsorted(rank, r)) + 1)


def build_tables(orc, rec, rank, n_item):
    """The device's tables for one user, restated: [(T_g, band_g)] per side."""
    S = len(rank)
    L = table_levels(S)
    capped = float(rec[4]) >= S - 1e-3
    out = []
    for side in (0, 1):
        T = orc.level_boundaries_at(rec, rank, n_item, L, side)
        T[E - 1] = -np.inf
        bands = np.zeros(E, np.float32)
        for g in range(E - 1):
            if L[g] >= S + 1:
                T[g] = -np.inf
            if not np.isfinite(T[g]) or capped:
                continue
            n = int(L[g]) if side else int(L[g]) - 1
            m = model_margin(rec)
            smin, smax = float(rec[6]), float(rec[5])
            f = lambda q: model_value(rec, side == 1, q)
            va, vb = f(smin), f(smax)
            if va < n - m or vb > n + m:
                continue
            zlo, zhi = smin, smax
            if va > n + m:
                lo, hi = smin, smax
                for _ in range(80):
                    mid = 0.5 * (lo + hi)
                    if mid <= lo or mid >= hi:
                        break
                    if f(mid) > n + m:
                        lo = mid
                    else:
                        hi = mid
                zlo = lo
            if vb < n - m:
                lo, hi = smin, smax
                for _ in range(80):
                    mid = 0.5 * (lo + hi)
                    if mid <= lo or mid >= hi:
                        break
                    if f(mid) >= n - m:
                        lo = mid
                    else:
                        hi = mid
                zhi = hi
            w = max(abs(float(T[g]) - zlo), abs(zhi - float(T[g])))
            bands[g] = np.nextafter(np.float32(w * (1 + 1e-6) + 1e-30), np.float32(np.inf))
        out.append((T.astype(np.float32), bands))
    return out


def f32_up(x):
    return np.nextafter(np.float32(x), np.float32(np.inf))


def f32_down(x):
    return np.nextafter(np.float32(x), np.float32(-np.inf))


def screen(T, band, q, dq):
    """lvt_screen: the coarse level #{g: q < T_g} and whether the table decides it for q +- dq."""
    c = 0
    for st in (8, 4, 2, 1):
        if q < T[c + st - 1]:
            c += st
    ok = True
    if c < E - 1:
        ok = float(f32_down(np.float32(q) - np.float32(dq))) >= float(f32_up(T[c] + band[c]))
    if c > 0:
        ok = ok and float(f32_up(np.float32(q) + np.float32(dq))) < float(f32_down(T[c - 1] - band[c - 1]))
    return c, ok


def users(orc, rng, S, n_item):
    rank = np.sort(rng.choice(np.arange(1, n_item - 1), S, replace=False)).astype(np.int32)
    recs = []
    for spread in (0.05, 0.2, 0.6):
        thr = -np.sort(-(rng.standard_normal((2, S)) * spread).astype(np.float32), axis=1)
        recs += list(orc.fit_regression(thr))
    steep = recs[0].copy()
    steep[3] = np.float32(0.01)  # a narrow CDF: boundaries crowd together
    capped = recs[1].copy()
    capped[4] = np.float32(S)
    return rank, recs + [steep, capped]


def test_reference_model_rounding_within_a_third_of_the_margin():
    """|v_reference - v| < margin / 3 over a dense grid of z and varied (a, b, err)."""
    orc = Oracle()
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(6):
        S = 512
        a = -float(rng.uniform(50, 2000))
        b = float(rng.uniform(-100, S + 100))
        err = float(rng.uniform(0.01, 30))
        rec = np.array([a, b, 0.0, 1.0, err, 10.0, -10.0], np.float32)
        for z in np.linspace(-7.5, 7.5, 6001).astype(np.float32):
            ix = float(orc.cdf_phi(z))
            pred = np.float32(np.float32(ix) * rec[0]) + rec[1]
            for upper in (False, True):
                v_ref = float(np.float32(pred - rec[4]) if upper else np.float32(pred + rec[4]))
                d = abs(v_ref - model_value(rec, upper, float(z)))
                worst = max(worst, d / model_margin(rec))
    assert worst < 1 / 3, worst
    print('worst fraction of the margin', worst)


@pytest.mark.parametrize("S,n_item", [(512, 17770), (64, 5000), (20, 5000)])
def test_table_screen_decides_the_oracle_coarse_level(S, n_item):
    orc = Oracle()
    rng = np.random.default_rng(S)
    rank, recs = users(orc, rng, S, n_item)
    for rec in recs:
        tabs = build_tables(orc, rec, rank, n_item)
        for side in (0, 1):
            T, band = tabs[side]
            assert np.all(T[1:] <= T[:-1])
            probes = list(rng.uniform(float(rec[6]) - 0.1, float(rec[5]) + 0.1, 60))
            for g in range(E - 1):
                if np.isfinite(T[g]):
                    t = np.float32(T[g])
                    w = max(float(band[g]), 1e-7)
                    probes += [t, f32_down(t), f32_up(t)] + list(t + np.float32(w) * np.linspace(-3, 3, 13))
            decided = 0
            for q in np.array(probes, np.float32):
                c, ok = screen(T, band, float(q), 0.0)
                if not ok:
                    continue
                decided += 1
                lv = level(orc, rec, rank, n_item, float(q), side)
                assert c == coarse(lv, S), (side, float(q), c, lv)
            assert decided > len(probes) // 3


def test_screen_leaves_every_band_undecided():
    """No score inside a boundary's guard band is decided from the table (the zone where the
    reference's rounding can put the level on either side), and scores just outside the bands of
    isolated boundaries are."""
    orc = Oracle()
    rng = np.random.default_rng(7)
    S, n_item = 512, 17770
    rank, recs = users(orc, rng, S, n_item)
    inside = outside = 0
    for rec in recs[:4]:
        tabs = build_tables(orc, rec, rank, n_item)
        for side in (0, 1):
            T, band = tabs[side]
            for g in range(E - 1):
                if not (np.isfinite(T[g]) and band[g] > 0):
                    continue
                for x in (-0.99, -0.5, 0.0, 0.5, 0.99):
                    _, ok = screen(T, band, float(T[g] + np.float32(band[g]) * np.float32(x)), 0.0)
                    assert not ok
                    inside += 1
                lo = T[g + 1] + band[g + 1] if np.isfinite(T[g + 1]) else -np.inf
                hi = T[g - 1] - band[g - 1] if g > 0 and np.isfinite(T[g - 1]) else np.inf
                for q in (T[g] - np.float32(2.5) * band[g], T[g] + np.float32(2.5) * band[g]):
                    if lo + band[g] < q < hi - band[g]:
                        _, ok = screen(T, band, float(q), 0.0)
                        assert ok
                        outside += 1
    assert inside > 0 and outside > 0


@pytest.mark.gpu
def test_device_tables_match_the_restatement():
    """The device's tables (rkr_index_level_tables) equal the restatement: boundaries bit for bit,
    guard bands to the double bisection's resolution (and never narrower by more than that)."""
    import rkr_b200
    orc = Oracle()
    rng = np.random.default_rng(21)
    S, n_item, d = 512, 17770, 8
    rank, recs = users(orc, rng, S, n_item)
    recs = np.stack(recs)
    user = orc.normalize(rng.standard_normal((recs.shape[0], d)).astype(np.float32))
    item = rng.standard_normal((n_item, d)).astype(np.float32)
    with rkr_b200.Index(user, item) as ix:
        ix.load_regression(rank, recs)
        levels, tab = ix.level_tables()
    assert np.array_equal(levels, table_levels(S))
    for u, rec in enumerate(recs):
        want = build_tables(orc, rec, rank, n_item)
        for side in (0, 1):
            T, band = want[side]
            assert np.array_equal(tab[u, side, :, 0].view(np.int32), T.view(np.int32)), (u, side)
            np.testing.assert_allclose(tab[u, side, :, 1], band, rtol=1e-5, atol=0)


# ---- the pair-scores kernel's upper side: monotone limits, a saturated count, a verification pair ----

def rd32(x):
    """x (a double) rounded down to binary32 (__fsub_rd / __fadd_rd of binary32 operands)."""
    r = np.float32(x)
    return f32_down(r) if float(r) > x else r


def ru32(x):
    r = np.float32(x)
    return f32_up(r) if float(r) < x else r


def verify_rows(T, band):
    """lvt_limits_row then lvt_verify_row (csrc/rkr_regression.cuh): entry c = (hi_c, lo_(c-1))."""
    lo = np.array([rd32(float(T[j]) - float(band[j])) for j in range(E)], np.float32)
    hi = np.array([ru32(float(T[j]) + float(band[j])) for j in range(E)], np.float32)
    if np.isnan(lo).any() or np.isnan(hi).any():
        return np.full((E, 2), np.nan, np.float32)
    lo = np.minimum.accumulate(lo)
    hi = np.maximum.accumulate(hi[::-1])[::-1]
    ver = np.empty((E, 2), np.float32)
    ver[:, 0] = hi
    ver[0, 1] = np.inf
    ver[1:, 1] = lo[:-1]
    return ver


def screen_directed(T, band, q, dq):
    """lvt_screen with the device's directed roundings (rd32 / ru32, exact where the result is)."""
    c = 0
    for st in (8, 4, 2, 1):
        if q < T[c + st - 1]:
            c += st
    qm, qp = rd32(float(np.float32(q)) - float(np.float32(dq))), ru32(float(np.float32(q)) + float(np.float32(dq)))
    ok = True
    if c < E - 1:
        ok = qm >= ru32(float(T[c]) + float(band[c]))
    if c > 0:
        ok = ok and qp < rd32(float(T[c - 1]) - float(band[c - 1]))
    return c, bool(ok)


def sat(x):
    return np.float32(0) if np.isnan(x) else np.float32(min(max(float(x), 0.0), 1.0))


def upper_screen(ver, q, dq, n_cache=10):
    """The kernel's upper side for bound score q, its distance dq: (decided, coarse level)."""
    f32 = np.float32
    qm, qp = rd32(float(f32(q)) - float(f32(dq))), ru32(float(f32(q)) + float(f32(dq)))
    with np.errstate(over="ignore", invalid="ignore"):
        cached = [f32(ver[g + 1, 1] * f32(2.0 ** 100)) for g in range(n_cache)]
        nq = f32(qp * f32(-2.0 ** 100))
        acc = [f32(0), f32(0)]
        for e in range(0, n_cache, 2):
            acc[0] = f32(acc[0] + sat(f32(cached[e] + nq)))
            acc[1] = f32(acc[1] + sat(f32(cached[e + 1] + nq)))
    c = int(np.rint(f32(acc[0] + acc[1])))
    ok = bool(qm >= ver[c, 0] and qp < ver[c, 1])
    if not ok and c == n_cache:
        k = 0
        for st in (8, 4, 2, 1):
            if qp < ver[k + st, 1]:
                k += st
        c, ok = k, bool(qm >= ver[k, 0] and qp < ver[k, 1])
    return ok, c


@pytest.mark.parametrize("S,n_item", [(512, 17770), (64, 5000)])
def test_upper_side_count_decides_within_the_table_screen(S, n_item):
    """Every pair the kernel's upper side decides has the oracle's coarse level, and lvt_screen decides
    it too, with the same level (the monotone limits only move outward); a verification pair accepts
    no level but the pair's own."""
    orc = Oracle()
    rng = np.random.default_rng(100 + S)
    rank, recs = users(orc, rng, S, n_item)
    decided = both = 0
    for rec in recs:
        T, band = build_tables(orc, rec, rank, n_item)[1]
        ver = verify_rows(T, band)
        probes = list(rng.uniform(float(rec[6]) - 0.1, float(rec[5]) + 0.1, 40))
        for g in range(E - 1):
            if np.isfinite(T[g]):
                t = np.float32(T[g])
                w = max(float(band[g]), 1e-7)
                probes += [t, f32_down(t), f32_up(t)] + list(t + np.float32(w) * np.linspace(-3, 3, 7))
        for q in np.array(probes, np.float32):
            for dq in (0.0, 1e-6, 1e-3):
                ok, c = upper_screen(ver, q, dq)
                c0, ok0 = screen_directed(T, band, float(q), dq)
                if ok0:
                    both += 1
                if not ok:
                    continue
                decided += 1
                assert ok0 and c == c0, (float(q), dq, c, c0, ok0)
                assert c == coarse(level(orc, rec, rank, n_item, float(q), 1), S)
                qm, qp = rd32(float(q) - dq), ru32(float(q) + dq)
                for c2 in range(E):
                    if c2 != c:
                        assert not (qm >= ver[c2, 0] and qp < ver[c2, 1]), (float(q), c, c2)
    assert decided > 0.9 * both, (decided, both)
