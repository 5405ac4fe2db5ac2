"""The -Ofast build of the reference harness (oracle/_ref/librkr_ref_fast.so), which bench.py times
beside the strict build: it must load and answer QSRPNormalLP::Retrieval on a small index built on
the host.  Its float sums may reassociate, so only the strict build is held to the oracle."""
import os

import numpy as np
import pytest

import rkr_b200 as R
from checkers import REF_FAST_SO, Oracle, Reference, ReferenceQsrp


@pytest.mark.skipif(not (Reference.available() and os.path.exists(REF_FAST_SO)),
                    reason="oracle/_ref not built (needs the reference sources)")
def test_fast_reference_build_answers():
    rng = np.random.default_rng(11)
    n_user, n_item, d, k = 600, 900, 24, 10
    O = Oracle()
    user = O.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = rng.standard_normal((n_item, d)).astype(np.float32)
    query = item[:12].copy()
    rank = np.unique(np.concatenate([np.arange(16), np.linspace(16, n_item - 2, 16).astype(int)])).astype(np.int32)
    thr = O.build_thresholds(user, item, rank)
    reg = R.fit_regression(thr)
    ti, su, cd = R.svd_build(user, 0.7)
    got = {}
    for name, so in (("strict", None), ("fast", REF_FAST_SO)):
        kw = {} if so is None else {"so": so}
        ref = ReferenceQsrp(user, su, ti, item, cd, rank, thr, rank, reg, 2, **kw)
        try:
            out, st, secs = ref.run(query, k)
        finally:
            ref.close()
        assert out.shape == (len(query), k) and secs >= 0.0
        assert np.all((out["user_id"] >= 0) & (out["user_id"] < n_user))
        got[name] = out
    want, _ = O.qsrp_retrieval(user, su, ti, item, cd, rank, thr, rank, reg, query, k)
    assert np.array_equal(np.ascontiguousarray(got["strict"]).view(np.int32), np.ascontiguousarray(want).view(np.int32))
