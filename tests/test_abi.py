"""CPU checks of the product library: it loads, exports every entry point include/rkr.h declares,
and its host-side build steps reproduce the reference (golden fixtures, oracle)."""
import os
import re

import numpy as np
import pytest

import rkr_b200
from checkers import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def header_functions():
    text = open(os.path.join(ROOT, "include", "rkr.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|int|void)\s*\**\s*(rkr_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 20
    assert sorted(rkr_b200.EXPORTS) == names
    for n in names:
        assert hasattr(rkr_b200.lib(), n), n
    assert rkr_b200.lib().rkr_version() >= 1


def load(case):
    return dict(np.load(os.path.join(GOLDEN, case + ".npz")))


@pytest.mark.parametrize("case", ["small", "fakenormal"])
def test_host_build_steps_match_reference(case):
    g = load(case)
    un = rkr_b200.normalize(g["user"])
    assert np.array_equal(un.view(np.int32), g["user_norm"].view(np.int32))
    si = rkr_b200.sample_item(g["item"].shape[0], g["sample_item"].shape[0])
    assert np.array_equal(si, g["sample_item"])
    kth, sid = rkr_b200.sort_kth_rank(g["accu"], int(g["sample_topk"]))
    assert np.array_equal(kth, g["sort_kth"]) and np.array_equal(sid, g["sort_sid"])
    opt, cost = rkr_b200.find_optimal_sample_rank(un.shape[0], g["item"].shape[0], g["opt_rank"].shape[0],
                                                 g["sort_kth"], g["accu"][g["sort_sid"]])
    assert np.array_equal(opt, g["opt_rank"]) and cost == int(g["opt_cost"])
    assert np.array_equal(rkr_b200.uniform_sample_rank(g["item"].shape[0], g["uni_rank"].shape[0]), g["uni_rank"])


@pytest.mark.parametrize("case", ["small", "fakenormal"])
def test_regression_fit_matches_reference(case):
    """mu, sigma, extremes bit-exact; (a, b, error) equal up to the LP solver's rounding (the
    reference's own fit is randomised); the fitted error covers every sample point."""
    g = load(case)
    rec = rkr_b200.fit_regression(g["thr"])
    ref = g["reg"]
    assert np.array_equal(rec[:, 2:4].view(np.int32), ref[:, 2:4].view(np.int32))
    assert np.array_equal(rec[:, 5:7].view(np.int32), ref[:, 5:7].view(np.int32))
    np.testing.assert_allclose(rec[:, 4], ref[:, 4], rtol=1e-5, atol=1e-4)
    np.testing.assert_allclose(rec[:, :2], ref[:, :2], rtol=1e-4, atol=1e-3)
    O = Oracle()
    S = g["thr"].shape[1]
    for u in range(0, rec.shape[0], 11):
        a, b, mu, sigma, err = (float(v) for v in rec[u, :5])
        for j in range(S - 1):
            for x in (O.cdf_phi((g["thr"][u, j] - mu) / sigma), O.cdf_phi((g["thr"][u, j + 1] - mu) / sigma)):
                assert abs(a * float(x) + b - (j + 1)) <= err + 1e-3


def test_svd_build_is_a_valid_transform():
    """transfer_user . (transfer_item q) == <user, q> and check_dim follows the sigma ratio."""
    g = load("small")
    ti, su, cd = rkr_b200.svd_build(g["user_norm"], 0.7)
    q = g["query"][:5].astype(np.float64)
    lhs = su.astype(np.float64) @ (ti.astype(np.float64) @ q.T)
    rhs = g["user_norm"].astype(np.float64) @ q.T
    np.testing.assert_allclose(lhs, rhs, atol=2e-4)
    assert 0 <= cd < g["user"].shape[1]


def test_invalid_arguments_raise():
    with pytest.raises(rkr_b200.RkrError):
        rkr_b200.uniform_sample_rank(10, 0)
    with pytest.raises(rkr_b200.RkrError):
        rkr_b200.sample_item(10, 11)
