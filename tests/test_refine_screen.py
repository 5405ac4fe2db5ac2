"""The decision arithmetic of the tensor-core refinement (csrc/rkr_refine_tc.cu), restated on the CPU:
candidates with their own power-of-two scale, items in groups of 8 under one scale, four signed
7-bit digits per coordinate, the digit products summed exactly per part (first check_dim
coordinates, the rest), the accumulators combined by three binary32 FMAs, and the six thresholds of
the reference's per-item test (RefineCPUIPBound::RefineRank, RefineCPUIPBound.hpp:93-150) formed
once per (candidate, group) with outward rounding and scaled to digit units.  Every test the screen
settles must come out as the reference's binary32 test does; the rest are listed for the exact path.
The US form (RefineCPU.hpp:33-55, count of ip > q over the unsplit score) is checked the same way."""
import numpy as np

from test_scores_screen import U24, fma32

KCOMB, KSIGMA, KSAFE = np.float32(1.8e-7), np.float32(1.3e-7), np.float32(1.0 + 1.0 / 65536.0)


def part_coef(n):
    if n <= 0:
        return np.float32(0), np.float32(0)
    g = n * U24 / (1.0 - n * U24)
    cn = np.float32(U24 * (1.0 + g) / (1.0 - U24) * 1.0001)
    ke = np.float32(n * (3.02 * 2.0 ** -30 + 2.0 ** -29 + 1.1e-4 * U24) * 1.01)
    return cn, ke


def exponent(mx):
    _, x = np.frexp(mx)
    return np.where(mx > 0, x + 1, 0).astype(np.int64)


def digits(rows, e):
    """Four signed 7-bit digits of rows scaled by 2^-e (e per row), as the slicing kernels cut them."""
    a = (rows * np.ldexp(np.float32(1), -e)[:, None].astype(np.float32)).astype(np.float32)
    out = []
    for _ in range(4):
        t = (a * np.float32(128)).astype(np.float32)
        d = np.rint(t).astype(np.float32)
        a = (t - d).astype(np.float32)
        out.append(d.astype(np.int64))
    assert all(np.abs(d).max() <= 64 for d in out)
    return out


def wnorm(x):
    n = x.shape[1]
    if n == 0:
        return np.zeros(x.shape[0])
    t = np.arange(n)
    w = np.where(t == 0, n, n - t + 1).astype(np.float64)
    return np.sqrt((w * x.astype(np.float64) ** 2).sum(axis=1) * (1 + 1e-12))


def up32(x):
    """float64 -> the smallest float32 >= x."""
    y = np.asarray(x, np.float64).astype(np.float32)
    return np.where(y.astype(np.float64) < x, np.nextafter(y, np.float32(np.inf)), y).astype(np.float32)


def down32(x):
    y = np.asarray(x, np.float64).astype(np.float32)
    return np.where(y.astype(np.float64) > x, np.nextafter(y, np.float32(-np.inf)), y).astype(np.float32)


def seq(a, b):
    """The reference's sequential binary32 sums of a_k b_k for every (row of a, row of b)."""
    s = np.zeros((a.shape[0], b.shape[0]), np.float32)
    for k in range(a.shape[1]):
        s = (s + (a[:, k:k + 1] * b[None, :, k]).astype(np.float32)).astype(np.float32)
    return s


def combine(acc):
    f = [x.astype(np.float32) for x in acc]  # exact: |acc| < 2^22
    return fma32(fma32(fma32(f[0], 128, f[1]), 128, f[2]), 128, f[3])


def screen(users, items, c, qv, ipbound):
    """(decided, cnt, und) per (candidate, item) as the kernel's epilogue settles them."""
    n_u, dim = users.shape
    n_i = items.shape[0]
    assert n_i % 8 == 0
    cu = c if ipbound else dim
    eu = exponent(np.abs(users).max(axis=1))
    mg = np.abs(items).reshape(n_i // 8, 8, dim).max(axis=(1, 2))
    eg = exponent(mg)
    ei = np.repeat(eg, 8)
    du, di = digits(users, eu), digits(items, ei)
    acc = lambda lo, hi: [sum(du[i][:, lo:hi] @ di[g - i][:, lo:hi].T for i in range(g + 1)) for g in range(4)]
    l = combine(acc(0, cu))
    r = combine(acc(cu, dim)) if cu < dim else np.zeros_like(l)
    cl, kl = part_coef(cu)
    cr, kr = part_coef(dim - cu)
    WLu, WRu = up32(wnorm(users[:, :cu])), up32(wnorm(users[:, cu:]))
    NLu, NRu = up32(np.linalg.norm(users[:, :cu].astype(np.float64), axis=1) * (1 + 1e-12)), \
        up32(np.linalg.norm(users[:, cu:].astype(np.float64), axis=1) * (1 + 1e-12))
    grp = lambda v: np.repeat(v.reshape(-1, 8).max(axis=1), 8)
    WLg, WRg = grp(up32(wnorm(items[:, :cu]))), grp(up32(wnorm(items[:, cu:])))
    NLg = grp(up32(np.linalg.norm(items[:, :cu].astype(np.float64), axis=1) * (1 + 1e-12)))
    NRg = grp(up32(np.linalg.norm(items[:, cu:].astype(np.float64), axis=1) * (1 + 1e-12)))
    # the reference's tail norms (row_norm_kernel: sqrt of the sequential binary32 sum of squares)
    rn = lambda x: np.sqrt(np.diagonal(seq(x[:, c:], x[:, c:])).astype(np.float32)).astype(np.float32)
    irn, un = rn(items), rn(users)
    IRg = grp(irn)
    Eu, Eg = np.ldexp(np.float32(1), eu).astype(np.float32), np.ldexp(np.float32(1), ei).astype(np.float32)
    EE = (Eu[:, None] * Eg[None, :]).astype(np.float32)
    nl = (NLu[:, None] * NLg[None, :]).astype(np.float32)
    cWL, cWR = (cl * WLu).astype(np.float32), (cr * WRu).astype(np.float32)
    DL = fma32(cWL[:, None], WLg[None, :], fma32(EE, kl, (KCOMB * nl).astype(np.float32)))
    inv = np.ldexp(np.float64(1), 35 - eu[:, None] - ei[None, :])
    qv2 = qv[:, None].astype(np.float32)
    if not ipbound:
        M = (fma32(KSIGMA, nl, DL) * KSAFE).astype(np.float32)
        t_hi = (up32(qv2.astype(np.float64) + M) * inv).astype(np.float32)
        t_lo = (down32(qv2.astype(np.float64) - M) * inv).astype(np.float32)
        cnt = l > t_hi
        decided = cnt | (l <= t_lo)
        return decided, cnt.astype(int), np.zeros_like(cnt, int)
    NRp = (NRu[:, None] * NRg[None, :]).astype(np.float32)
    DR = fma32(cWR[:, None], WRg[None, :], fma32(EE, kr, (KCOMB * NRp).astype(np.float32)))
    Ms = (fma32(KSIGMA, fma32(un[:, None], IRg[None, :], nl), DL) * KSAFE).astype(np.float32)
    Mt = (fma32(KSIGMA, fma32(NRu[:, None], NRg[None, :], nl), (DL + DR).astype(np.float32)) * KSAFE).astype(np.float32)
    lowq, highq = (qv2 - np.float32(8e-3)).astype(np.float32), (qv2 + np.float32(8e-3)).astype(np.float32)
    sc = lambda x: (x.astype(np.float64) * inv).astype(np.float32)  # exact: a power of two
    t_sk, t_ns = sc(down32(lowq.astype(np.float64) - Ms)), sc(up32(lowq.astype(np.float64) + Ms))
    t_ct, t_fu = sc(up32(highq.astype(np.float64) + Ms)), sc(down32(highq.astype(np.float64) - Ms))
    t_hi, t_mi = sc(up32(qv2.astype(np.float64) + Mt)), sc(down32(qv2.astype(np.float64) - Mt))
    un_s = sc(np.broadcast_to(un[:, None], l.shape))
    rt = (irn[None, :] * un_s).astype(np.float32)
    s, d, t = (l + rt).astype(np.float32), (l - rt).astype(np.float32), (l + r).astype(np.float32)
    sk = s < t_sk
    ns = s >= t_ns
    c1 = ns & (d > t_ct)
    f1 = ns & ~c1 & (d <= t_fu)
    hi, mi = t >= t_hi, t < t_mi
    decided = sk | c1 | (f1 & (hi | mi))
    cnt = (~sk & (c1 | (f1 & hi))).astype(int)
    und = (~sk & f1).astype(int)
    return decided, cnt, und


def reference(users, items, c, qv, ipbound):
    if not ipbound:
        full = seq(users, items)
        return (full > qv[:, None].astype(np.float32)).astype(int), np.zeros(full.shape, int)
    left, rest = seq(users[:, :c], items[:, :c]), seq(users[:, c:], items[:, c:])
    rn = lambda x: np.sqrt(np.diagonal(seq(x[:, c:], x[:, c:])).astype(np.float32)).astype(np.float32)
    right = (rn(users)[:, None] * rn(items)[None, :]).astype(np.float32)
    q = qv[:, None].astype(np.float32)
    lowq, highq = (q - np.float32(8e-3)).astype(np.float32), (q + np.float32(8e-3)).astype(np.float32)
    skip = lowq > (left + right).astype(np.float32)
    counted = ~skip & (highq < (left - right).astype(np.float32))
    full = ~skip & ~counted
    hit = (left + rest).astype(np.float32) >= q
    return (counted | (full & hit)).astype(int), full.astype(int)


def engine_rows(seed, n_u=48, n_i=256, dim=150):
    rng = np.random.default_rng(seed)
    users = rng.standard_normal((n_u, dim)).astype(np.float32)
    users = (users / np.sqrt((users.astype(np.float64) ** 2).sum(axis=1, keepdims=True))).astype(np.float32)
    items = (rng.standard_normal((n_i, dim)) / np.sqrt(dim) * np.exp(rng.normal(0, 0.3, (n_i, 1)))).astype(np.float32)
    # items in the norm order, as the engine stores them
    order = np.argsort(-np.linalg.norm(items.astype(np.float64), axis=1), kind="stable")
    return users, items[order]


def check(users, items, c, qv, ipbound, max_listed):
    dec, cnt, und = screen(users, items, c, qv, ipbound)
    rc, ru = reference(users, items, c, qv, ipbound)
    assert np.array_equal(cnt[dec], rc[dec]), "a settled count differs from the reference's"
    if ipbound:
        # und is settled by the bound tests alone (also for pairs listed for their count)
        _, _, und_all = screen(users, items, c, qv, ipbound)
        settled_und = dec | (und_all == 1)
        assert np.array_equal(und_all[settled_und], ru[settled_und])
    frac = 1.0 - dec.mean()
    assert frac <= max_listed, frac
    return frac


def test_refine_screen_matches_reference_split():
    for c in (104, 30):
        users, items = engine_rows(1)
        full = seq(users, items)
        rng = np.random.default_rng(2)
        # thresholds at the scores of random items (the candidates' own query scores are such values)
        qv = full[np.arange(users.shape[0]), rng.integers(0, items.shape[0], users.shape[0])]
        check(users, items, c, qv, True, 0.02)


def test_refine_screen_exact_ties_are_listed_or_right():
    users, items = engine_rows(3)
    c = 104
    left, rest = seq(users[:, :c], items[:, :c]), seq(users[:, c:], items[:, c:])
    tot = (left + rest).astype(np.float32)
    j = np.random.default_rng(4).integers(0, items.shape[0], users.shape[0])
    for qv in (tot[np.arange(users.shape[0]), j],                                  # exact ties
               np.nextafter(tot[np.arange(users.shape[0]), j], np.float32(np.inf)),  # one ulp above
               np.nextafter(tot[np.arange(users.shape[0]), j], np.float32(-np.inf))):
        check(users, items, c, qv.astype(np.float32), True, 0.05)


def test_refine_screen_us_form():
    users, items = engine_rows(5)
    full = seq(users, items)
    j = np.random.default_rng(6).integers(0, items.shape[0], users.shape[0])
    qv = full[np.arange(users.shape[0]), j]
    check(users, items, 150, qv, False, 0.02)


def test_refine_screen_detects_a_margin_too_small(monkeypatch):
    """The check has teeth: the same restatement with its margins 1000x too small settles some tests
    against the reference's outcome (the planted error lives in this CPU restatement only)."""
    import test_refine_screen as T
    users, items = engine_rows(1)
    c = 104
    tot = (seq(users[:, :c], items[:, :c]) + seq(users[:, c:], items[:, c:])).astype(np.float32)
    qv = tot[np.arange(users.shape[0]), np.random.default_rng(4).integers(0, items.shape[0], users.shape[0])]
    orig = T.part_coef
    monkeypatch.setattr(T, "KSAFE", np.float32(1e-3))
    monkeypatch.setattr(T, "KSIGMA", np.float32(0))
    monkeypatch.setattr(T, "KCOMB", np.float32(0))
    monkeypatch.setattr(T, "part_coef", lambda n: tuple(np.float32(x * 1e-3) for x in orig(n)))
    dec, cnt, _ = T.screen(users, items, c, qv, True)
    rc, _ = T.reference(users, items, c, qv, True)
    assert int((cnt[dec] != rc[dec]).sum()) > 0
