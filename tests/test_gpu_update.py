"""User insertion and deletion against a built index (rkr_index_insert_users / rkr_index_delete_users,
QSRPNormalLPUpdate::InsertUser / DeleteUser): after each update the index answers as the oracle does
on the updated user set -- the appended users' thresholds and models as a full build computes them,
the transform rebuilt over every user after an insertion and kept after a deletion, and the carried
QSRPNormalLP scores resized as the reference resizes its vector (zeros appended; after a deletion
the first n_user entries stay)."""
import numpy as np
import pytest

import rkr_b200 as R
from checkers import Oracle

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.int32).reshape(-1)


@pytest.fixture(scope="module")
def data():
    rng = np.random.default_rng(2024)
    d, n_item = 32, 3000
    a = R.normalize(rng.standard_normal((3000, d)).astype(np.float32))
    b = R.normalize(rng.standard_normal((1500, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, 24), np.linspace(24, n_item - 2, 40).astype(int)])).astype(np.int32)
    q = [item[rng.choice(n_item, 30, replace=False)].copy() for _ in range(3)]
    dele = rng.choice(4500, 700, replace=False).astype(np.int64)
    return dict(a=a, b=b, item=item, rank=rank, q=q, dele=dele)


def test_insert_then_delete_users_answers_as_the_oracle(data):
    orc = Oracle()
    a, b, item, rank, q, k = data["a"], data["b"], data["item"], data["rank"], data["q"], 20
    with R.Index(a, item) as ix:
        thr_a = ix.build_sample_search(rank)
        reg_a = ix.fit_regression()
        ti, su, cd = ix.svd_build(0.7)
        state = np.zeros(a.shape[0], np.float32)
        out = ix.retrieval("QSRPNormalLP", q[0], k)
        want, _ = orc.qsrp_retrieval(a, su, ti, item, cd, rank, thr_a, rank, reg_a, q[0], k, state)
        assert np.array_equal(bits(out), bits(want))
        # insertion: thresholds and models of the new users, the transform over all users
        ix.insert_users(b, 0.7)
        ab = np.concatenate([a, b])
        thr_ab = orc.build_thresholds(ab, item, rank)
        reg_ab = R.fit_regression(thr_ab)
        ti2, su2, cd2 = ix.svd_read()
        assert su2.shape[0] == ab.shape[0]
        state = np.concatenate([state, np.zeros(b.shape[0], np.float32)])
        out = ix.retrieval("QSRPNormalLP", q[1], k)
        want, _ = orc.qsrp_retrieval(ab, su2, ti2, item, cd2, rank, thr_ab, rank, reg_ab, q[1], k, state)
        assert np.array_equal(bits(out), bits(want))
        out = ix.retrieval("QS", q[1], k)
        want, _ = orc.qs_retrieval(ab, item, cd2, rank, thr_ab, q[1], k)
        assert np.array_equal(bits(out), bits(want))
        # deletion: the rows of the others close up, the transform stays, the carried scores truncate
        ix.delete_users(data["dele"])
        keep = np.setdiff1d(np.arange(ab.shape[0]), data["dele"])
        state = state[:keep.size].copy()
        out = ix.retrieval("QSRPNormalLP", q[2], k)
        want, _ = orc.qsrp_retrieval(ab[keep], su2[keep], ti2, item, cd2, rank, thr_ab[keep], rank, reg_ab[keep],
                                     q[2], k, state)
        assert np.array_equal(bits(out), bits(want))
        ti3, su3, cd3 = ix.svd_read()
        assert np.array_equal(bits(su3), bits(su2[keep])) and cd3 == cd2


def test_updates_are_checked(data):
    a, item, rank = data["a"], data["item"], data["rank"]
    with R.Index(a[:500], item) as ix:
        with pytest.raises(R.RkrError):
            ix.insert_users(a[500:600])          # no thresholds yet
        ix.build_sample_search(rank)
        with pytest.raises(R.RkrError):
            ix.delete_users(np.array([3, 3]))    # a user twice
        with pytest.raises(R.RkrError):
            ix.delete_users(np.arange(500))      # every user
        ix.insert_users(a[500:600])
        assert ix.n_user == 600
        ix.delete_users(np.array([0, 599]))
        assert ix.n_user == 598
