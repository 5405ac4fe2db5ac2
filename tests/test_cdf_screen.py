"""The float-only CDF the device uses to screen regression levels stays within 1e-6 of the
reference's CDFPhi (NormalLinearRegressionLP.hpp:123-143) -- the bound the screen's margin
(|a| * 4e-6 + 8 ulp) relies on.  Swept on the CPU over a dense grid and the awkward regions
(tiny arguments, the tails)."""
import numpy as np

from checkers import Oracle


def cdf_f32(x):
    x = np.asarray(x, dtype=np.float32)
    a1, a2, a3 = np.float32(0.254829592), np.float32(-0.284496736), np.float32(1.421413741)
    a4, a5, p = np.float32(-1.453152027), np.float32(1.061405429), np.float32(0.3275911)
    sign = np.where(x < 0, np.float32(-1), np.float32(1))
    z = np.abs(x) / np.float32(1.41421354)
    t = np.float32(1) / (np.float32(1) + p * z)
    pt = (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t
    y = np.float32(1) - pt * np.exp(-z * z, dtype=np.float32)
    return (np.float32(0.5) * (np.float32(1) + sign * y)).astype(np.float32)


def test_float_cdf_within_1e6_of_reference():
    orc = Oracle()
    xs = np.concatenate([np.linspace(-12, 12, 200001), np.geomspace(1e-9, 1e-2, 5001),
                         -np.geomspace(1e-9, 1e-2, 5001), np.random.default_rng(0).normal(0, 3, 50000)])
    xs = xs.astype(np.float32)
    ref = np.array([orc.cdf_phi(v) for v in xs], dtype=np.float64)
    got = cdf_f32(xs).astype(np.float64)
    assert np.max(np.abs(got - ref)) < 1e-6
