"""The regression-level screen of the pair-scores kernel (level_side in csrc/rkr_scores_tc.cu), restated
on the CPU in binary32: for a bound score q known to within dq of the reference's, a side it settles
must give the level of the reference's ComputeRankBound (NormalLinearRegressionLP.hpp:326-380, through
the oracle) for every score within q +- dq -- across the CDF table's cells, near-integer predictions,
the extreme-score shortcuts (smax / smin) and users whose fit error reaches the cap."""
import numpy as np

from checkers import Oracle
from test_scores_screen import cdf_table

KCDF_TAB_ERR = np.float32(1.0e-6)
MARGIN_SCALE = 1.0  # 1 in level_side; the planted-error test shrinks it


def fma32(a, b, c):
    """binary32 fma of scalars: the product is exact in double; the sum's double rounding is far
    below the margins checked here."""
    return np.float32(float(a) * float(b) + float(c))


def level_side(rec, err_cap, S, q, dq, upper, tab):
    """(decided, level) as level_side computes them; rec = (a, b, mu, sigma, err, smax, smin)."""
    a, b, mu, sigma, err, smax, smin = [np.float32(x) for x in rec]
    f32 = np.float32
    inv_sigma = f32(1) / sigma                      # __frcp_rn
    capped = float(err) >= err_cap
    margin0 = f32(np.inf) if capped else \
        f32(f32(abs(a) * KCDF_TAB_ERR) + f32(f32(abs(a) + abs(b)) + abs(err)) * f32(4.8e-7)) + f32(1e-6)
    cu = f32(f32(abs(a) * inv_sigma) * f32(1.0001))
    q, dq = f32(q), f32(dq)
    z = f32(f32(q - mu) * inv_sigma)
    tv, td, th = tab
    # the table lookup of level_side: cell i, offset f in it, quadratic in Newton form
    t = min(max(fma32(z, f32(128), f32(1024)), f32(0)), f32(2047))
    tu = f32(f32(t - f32(0.5)) + f32(12582912.0))
    i = int(np.array([tu], np.float32).view(np.int32)[0] - 0x4B400000)
    fr = f32(t - f32(tu - f32(12582912.0)))
    cdf = fma32(fr, fma32(f32(fr - f32(1)), th[i], td[i]), tv[i])
    base = fma32(cdf, a, b)
    v = f32(base - err) if upper else f32(base + err)
    margin = f32(fma32(f32(cu * dq), fma32(td[i], f32(141), f32(1e-6)), margin0) * f32(MARGIN_SCALE))
    above = f32(q - dq) > smax
    below = f32(q + dq) < smin
    inside = f32(q + dq) <= smax and f32(q - dq) >= smin
    fl = f32(np.floor(v))
    frac = f32(v - fl)
    cv = fl if upper else (f32(fl + 1) if frac > 0 else fl)
    low = 0 if upper else 1
    lv_model = S + 1 if cv >= S else (low if cv < 0 else int(cv) + 1)
    in_lvl = (0 if upper else S + 1) if capped else lv_model
    if upper:
        lvl = 0 if above else (S if below else in_lvl)
    else:
        lvl = 1 if above else (S + 1 if below else in_lvl)
    decided_in = capped or (min(frac, f32(1) - frac) > margin and abs(v) < 1.6e7)
    ok = (above or below or (inside and decided_in)) and f32(dq * inv_sigma) <= f32(9.765625e-4)
    return ok, lvl


def level_rank(lvl, rank, S, n_item):
    return 0 if lvl == 0 else (n_item if lvl > S else int(rank[lvl - 1]))


def check_user(orc, rec, rank, n_item, S, qs, dqs, tab, rng):
    settled = total = 0
    err_cap = S - 1e-3
    reg = np.asarray(rec, np.float32)[None, :]
    for q in qs:
        for dq in dqs:
            for upper in (False, True):
                ok, lvl = level_side(rec, err_cap, S, q, dq, upper, tab)
                total += 1
                if not ok:
                    continue
                settled += 1
                want = level_rank(lvl, rank, S, n_item)
                lo, hi = np.float64(q) - dq, np.float64(q) + dq
                xs = np.unique(np.concatenate([[q], np.float32([lo, hi]), rng.uniform(lo, hi, 3)]).astype(np.float32))
                xs = xs[(xs.astype(np.float64) >= lo) & (xs.astype(np.float64) <= hi)]
                for x in xs:
                    lb, ub = orc.regression_rank_bound(reg, rank, n_item, [0], [x], [x])
                    got = int(ub[0]) if upper else int(lb[0])
                    assert got == want, (rec, q, dq, upper, x, got, want)
    return settled, total


def test_level_screen_agrees_with_reference():
    orc = Oracle()
    tab = cdf_table()
    rng = np.random.default_rng(9)
    n_item, S = 5000, 64
    rank = np.unique(np.concatenate([np.arange(1, 40), np.linspace(40, n_item - 2, S).astype(int)]))[:S]
    rank = np.sort(rank).astype(np.int32)
    thr = -np.sort(-(rng.standard_normal((24, S)) * rng.uniform(0.05, 0.5, (24, 1))).astype(np.float32), axis=1)
    reg = orc.fit_regression(thr)
    settled = total = 0
    for u in range(reg.shape[0]):
        rec = reg[u]
        smax, smin = float(rec[5]), float(rec[6])
        span = smax - smin
        qs = np.concatenate([rng.uniform(smin - 0.1 * span, smax + 0.1 * span, 60), [smax, smin]]).astype(np.float32)
        # uncertainties like the engine's (a few 1e-7 of the score): counted for coverage
        s, t = check_user(orc, rec, rank, n_item, S, qs, [0.0, 1e-7, 1e-6, 1e-5], tab, rng)
        settled += s
        total += t
        # past the screen's range (dq / sigma > 2^-10) it must leave the side to the exact path
        check_user(orc, rec, rank, n_item, S, qs[:10], [1e-3 * span], tab, rng)
    assert settled > 0.9 * total, (settled, total)  # the screen decides the great majority


def near_integer_scores(orc, rec, S, step=1):
    """Scores whose prediction pred -+ err lands on an integer (by bisection on the oracle's CDF),
    with their float neighbours."""
    a, b, mu, sigma, err = [float(x) for x in rec[:5]]
    qs = []
    for m in range(1, S - 1, step):
        for sgn in (1.0, -1.0):
            cdf_target = (m - b - sgn * err) / a
            if 0.0 < cdf_target < 1.0:
                lo, hi = -8.0, 8.0
                for _ in range(60):
                    mid = 0.5 * (lo + hi)
                    if orc.cdf_phi(np.float32(mid)) < cdf_target:
                        lo = mid
                    else:
                        hi = mid
                q0 = np.float32(mu + sigma * lo)
                qs += [q0, np.nextafter(q0, np.float32(np.inf)), np.nextafter(q0, np.float32(-np.inf))]
    return np.array(qs, np.float32)


def test_level_screen_capped_user_and_near_integers():
    orc = Oracle()
    tab = cdf_table()
    rng = np.random.default_rng(10)
    n_item, S = 5000, 64
    rank = np.linspace(1, n_item - 2, S).astype(np.int32)
    thr = -np.sort(-(rng.standard_normal((4, S)) * 0.2).astype(np.float32), axis=1)
    reg = orc.fit_regression(thr)
    # a user whose fit error reaches the cap takes the capped levels inside [smin, smax]
    capped = reg[0].copy()
    capped[4] = np.float32(S)
    qs = np.linspace(float(capped[6]) - 0.01, float(capped[5]) + 0.01, 41).astype(np.float32)
    check_user(orc, capped, rank, n_item, S, qs, [0.0, 1e-6], tab, rng)
    # scores whose prediction lands within a few ulps of an integer: settled only when right
    check_user(orc, reg[1], rank, n_item, S, near_integer_scores(orc, reg[1], S, 5), [0.0, 1e-7], tab, rng)


def test_level_screen_detects_a_missing_margin(monkeypatch):
    """The check has teeth: without its margin the restated screen settles some near-integer sides
    against the reference (the planted error lives in this CPU restatement only)."""
    import test_level_screen as T
    monkeypatch.setattr(T, "MARGIN_SCALE", 0.0)
    orc = Oracle()
    tab = cdf_table()
    rng = np.random.default_rng(10)
    n_item, S = 5000, 64
    rank = np.linspace(1, n_item - 2, S).astype(np.int32)
    thr = -np.sort(-(rng.standard_normal((4, S)) * 0.2).astype(np.float32), axis=1)
    reg = orc.fit_regression(thr)
    wrong = 0
    for u in range(reg.shape[0]):
        for q in near_integer_scores(orc, reg[u], S):
            for upper in (False, True):
                ok, lvl = T.level_side(reg[u], S - 1e-3, S, q, 0.0, upper, tab)
                lb, ub = orc.regression_rank_bound(reg[u][None, :], rank, n_item, [0], [q], [q])
                wrong += ok and (int(ub[0]) if upper else int(lb[0])) != level_rank(lvl, rank, S, n_item)
    assert wrong > 0
