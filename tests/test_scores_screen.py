"""The digit arithmetic of the tensor-core pair scores (csrc/rkr_scores_tc.cu), restated on the CPU:
rows split into four signed 7-bit digits under a power-of-two scale, the ten digit products with
i + j <= 5 summed exactly (as the int8 MMAs with int32 accumulation do), the four accumulators
combined by three binary32 FMAs.  The combined score must lie within the kernel's bound of the
reference's sequential binary32 sum (the sum the screen stands in for) on every pair, for the
distributions the engine sees (normalised users, lognormal-scaled items) and for awkward rows (wide
dynamic range, zeros, single spikes)."""
import numpy as np

U24 = 2.0 ** -24


def digits(rows):
    """Per row: (e, digits [4][n] int64) with |row| < 2^(e-1) and row = 2^e sum d_i 2^-7i + r."""
    rows = np.asarray(rows, np.float32)
    mx = np.max(np.abs(rows), axis=1)
    _, x = np.frexp(mx)
    e = np.where(mx > 0, x + 1, 0).astype(np.int64)
    a = (rows * np.ldexp(np.float32(1), -e)[:, None].astype(np.float32)).astype(np.float32)
    out = []
    for _ in range(4):
        t = (a * np.float32(128)).astype(np.float32)
        d = np.rint(t).astype(np.float32)
        a = (t - d).astype(np.float32)
        out.append(d.astype(np.int64))
    assert all(np.abs(d).max() <= 64 for d in out)
    return e, np.stack(out)


def fma32(a, b, c):
    """binary32 fma: the exact a * b + c (exact in binary64 here) rounded once."""
    return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)


def tc_score(da, ea, db, eb):
    acc = [sum(da[i] @ db[j].T for i in range(4) for j in range(4) if i + j == g) for g in range(4)]
    for x in acc:
        assert np.abs(x).max() < 2 ** 22
    f = [x.astype(np.float32) for x in acc]  # exact below 2^22
    v = fma32(fma32(fma32(f[0], 128, f[1]), 128, f[2]), 128, f[3])
    return (v.astype(np.float64) * np.ldexp(1.0, ea[:, None] + eb[None, :] - 35)).astype(np.float32)


def ref_seq(a, b):
    s = np.zeros((a.shape[0], b.shape[0]), np.float32)
    for k in range(a.shape[1]):
        s = (s + (a[:, k:k + 1] * b[None, :, k]).astype(np.float32)).astype(np.float32)
    return s


def wnorm(x):
    """Position-weighted norm of the rows: (sum_t w_t x_t^2)^(1/2), w_1 = n, w_t = n - t + 2."""
    n = x.shape[1]
    t = np.arange(n)
    w = np.where(t == 0, n, n - t + 1).astype(np.float64)
    return np.sqrt((w * x.astype(np.float64) ** 2).sum(axis=1))


def bound(a, ea, b, eb, n):
    gamma = n * U24 / (1 - n * U24)
    cn = U24 * (1 + gamma) / (1 - U24) * 1.0001
    ke = n * (3.02 * 2.0 ** -30 + 2.0 ** -29 + 1.1e-4 * U24) * 1.01
    return cn * np.outer(wnorm(a), wnorm(b)) + ke * np.ldexp(1.0, ea[:, None] + eb[None, :])


def check(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ea, da = digits(a)
    eb, db = digits(b)
    got = tc_score(da, ea, db, eb).astype(np.float64)
    ref = ref_seq(a, b).astype(np.float64)
    d = bound(a, ea, b, eb, a.shape[1]) + 1.8e-7 * np.abs(got)  # the combination's leading term, per pair
    err = np.abs(got - ref)
    assert np.all(err <= d), float(np.max(err / d))
    return float(np.max(err / d))


def test_bound_holds_on_engine_distributions():
    rng = np.random.default_rng(3)
    for n in (30, 50, 100, 150, 240):
        users = rng.standard_normal((64, n)).astype(np.float32)
        users /= np.linalg.norm(users, axis=1, keepdims=True)
        items = (rng.standard_normal((48, n)) / np.sqrt(n) * np.exp(rng.normal(0, 0.3, (48, 1)))).astype(np.float32)
        ratio = check(users, items)
        assert ratio < 0.5  # the bound is rigorous, and not so loose that the screen stops deciding


def test_bound_holds_on_adversarial_sums():
    """Sums whose roundings all push one way: equal-sign products, a large leading term then small
    ones, and decreasing magnitudes -- the cases the position weights are about."""
    rng = np.random.default_rng(5)
    n = 150
    pos = np.abs(rng.standard_normal((32, n))).astype(np.float32)
    lead = np.abs(rng.standard_normal((16, n))).astype(np.float32) * 1e-3
    lead[:, 0] = 1.0
    decay = (np.abs(rng.standard_normal((16, n))) * np.exp(-np.arange(n) / 20.0)).astype(np.float32)
    ones = np.ones((4, n), np.float32) * np.float32(1 / 3)
    rows = np.concatenate([pos, lead, decay, ones])
    check(rows, rows)
    check(rows, np.abs(rng.standard_normal((24, n))).astype(np.float32))


def test_bound_holds_on_awkward_rows():
    rng = np.random.default_rng(4)
    n = 64
    wide = (rng.standard_normal((16, n)) * np.exp(rng.uniform(-20, 20, (16, n)))).astype(np.float32)
    spikes = np.zeros((8, n), np.float32)
    spikes[np.arange(8), rng.integers(0, n, 8)] = rng.standard_normal(8).astype(np.float32) * 1e3
    zeros = np.zeros((2, n), np.float32)
    tiny = (rng.standard_normal((8, n)) * 1e-9).astype(np.float32)
    rows = np.concatenate([wide, spikes, zeros, tiny])
    other = np.concatenate([rng.standard_normal((16, n)).astype(np.float32), tiny, spikes])
    check(rows, other)
    check(other, rows)


def phi_as(z):
    """The reference's CDF formula (Abramowitz & Stegun 7.1.26) in double."""
    a1, a2, a3, a4, a5, p = 0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429, 0.3275911
    x = np.abs(z) / np.sqrt(2.0)
    t = 1.0 / (1.0 + p * x)
    y = 1.0 - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * np.exp(-x * x)
    return 0.5 * (1.0 + np.where(z < 0, -1.0, 1.0) * y)


def cdf_table():
    """The regression CDF table of the tensor-core screen: at z_i = -8 + i / 128 the value, the first
    difference and half the second difference, rounded to binary32."""
    z0 = -8.0 + np.arange(2048) / 128.0
    v0, v1, v2 = phi_as(z0), phi_as(z0 + 1.0 / 128.0), phi_as(z0 + 2.0 / 128.0)
    return v0.astype(np.float32), (v1 - v0).astype(np.float32), (0.5 * (v2 - 2 * v1 + v0)).astype(np.float32)


def cdf_tab_f32(z, tv, td, th):
    """The device's lookup, step by step in binary32 (fma as one rounding of the exact value)."""
    z = np.asarray(z, np.float32)
    t = fma32(z, np.float32(128), np.float32(1024))
    t = np.minimum(np.maximum(t, np.float32(0)), np.float32(2047))
    tu = ((t - np.float32(0.5)).astype(np.float32) + np.float32(12582912.0)).astype(np.float32)
    i = (tu.view(np.int32) - 0x4B400000).astype(np.int64)
    f = (t - (tu - np.float32(12582912.0)).astype(np.float32)).astype(np.float32)
    assert i.min() >= 0 and i.max() <= 2047 and f.min() >= -2.0 ** -14 and f.max() <= 1 + 2.0 ** -14
    inner = fma32((f - np.float32(1)).astype(np.float32), th[i], td[i])
    return fma32(f, inner, tv[i])


def test_cdf_table_within_bound_of_reference():
    """kCdfTabErr = 1e-6 in rkr_scores_tc.cu: the interpolated table against the reference's CDFPhi
    at the same argument, on a dense grid, the tails and tiny arguments."""
    from checkers import Oracle
    orc = Oracle()
    tv, td, th = cdf_table()
    zs = np.concatenate([np.linspace(-12, 12, 400001), np.geomspace(1e-9, 1e-2, 3001), -np.geomspace(1e-9, 1e-2, 3001),
                         np.random.default_rng(1).normal(0, 3, 30000)]).astype(np.float32)
    ref = np.array([orc.cdf_phi(v) for v in zs], dtype=np.float64)
    got = cdf_tab_f32(zs, tv, td, th).astype(np.float64)
    assert np.max(np.abs(got - ref)) < 8e-7  # the remaining 2e-7: the argument's few ulps


def test_cdf_table_density_bound():
    """The screen's slope bound: on each cell widened by 2^-10 on both sides, the formula's slope stays
    below D * 141 + 1e-6 (D the cell's stored difference)."""
    tv, td, th = cdf_table()
    phi = phi_as

    w = 2.0 ** -10
    for i in range(0, 2048, 1):
        z0 = -8.0 + i / 128.0
        zz = np.linspace(z0 - w, z0 + 1 / 128.0 + w, 41)
        h = 1e-7
        slope = np.max(np.abs(phi(zz + h) - phi(zz - h)) / (2 * h))
        assert slope <= td[i] * 141.0 + 1e-6, (i, slope, td[i] * 141.0)


def test_bound_detects_a_margin_too_small():
    """The check has teeth: the same sums against the bound scaled by 1e-3 leave some estimate outside
    it (the planted error lives in this CPU restatement only)."""
    rng = np.random.default_rng(5)
    n = 150
    a = np.abs(rng.standard_normal((32, n))).astype(np.float32)
    b = np.abs(rng.standard_normal((24, n))).astype(np.float32)
    ea, da = digits(a)
    eb, db = digits(b)
    got = tc_score(da, ea, db, eb).astype(np.float64)
    ref = ref_seq(a, b).astype(np.float64)
    d = (bound(a, ea, b, eb, n) + 1.8e-7 * np.abs(got)) * 1e-3
    assert np.any(np.abs(got - ref) > d)
