"""The threshold build that allocates nothing (rkr_build_thresholds_static).

It exists for callers that cannot let a library allocate device memory -- services that fix
their footprint at start-up, code under a caching allocator or a carved-up pool.  Its scratch is a
fixed array inside librkr_b200.so shared by every call, so this test checks, through the C ABI,
that two calls in a row -- with different problem sizes, so stale scratch from the first call
would show -- each give exactly the thresholds of the allocating entry point
(rkr_index_build_sample_search).  Thresholds are order statistics of exact float scores, so the
comparison is bit for bit.  This file is collected last on purpose.
"""
import numpy as np
import pytest

import rkr_b200

pytestmark = pytest.mark.gpu


def case(seed, n_user, n_item, d, n_sample):
    rng = np.random.default_rng(seed)
    user = rkr_b200.normalize(rng.standard_normal((n_user, d)).astype(np.float32))
    item = (rng.standard_normal((n_item, d)) * np.exp(rng.normal(0, 0.3, (n_item, 1)))).astype(np.float32)
    rank = np.unique(np.concatenate([np.arange(0, n_sample // 2),
                                     np.linspace(n_sample // 2, n_item - 1, n_sample - n_sample // 2).astype(int)]))
    return user, item, rank.astype(np.int32)


def test_static_threshold_build_matches_allocating_build_twice():
    import torch
    torch.cuda.set_device(0)
    # the first case needs several row batches of the 32 MiB scratch; the second is smaller, so
    # rows left over from the first call would corrupt it if the scratch were not fully rewritten
    for seed, shape in ((41, (3500, 4999, 48, 96)), (42, (700, 1203, 30, 40))):
        n_user, n_item, d, n_sample = shape
        user, item, rank = case(seed, n_user, n_item, d, n_sample)
        with rkr_b200.Index(user, item, device=0) as ix:
            want = ix.build_sample_search(rank)
        du = torch.from_numpy(user).cuda()
        di = torch.from_numpy(item).cuda()
        out = torch.full((n_user, rank.shape[0]), float("nan"), dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rkr_b200.build_thresholds_static(du.data_ptr(), n_user, di.data_ptr(), n_item, d, rank, out.data_ptr(),
                                         stream)
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.int32), want.view(np.int32)), f"mismatch for shape {shape}"


def test_static_threshold_build_rejects_oversize():
    import torch
    du = torch.zeros((4, 8), dtype=torch.float32, device="cuda")
    di = torch.zeros((20000, 8), dtype=torch.float32, device="cuda")
    out = torch.zeros((4, 17000), dtype=torch.float32, device="cuda")
    too_many = np.arange(17000, dtype=np.int32)  # above the 16384-rank maximum
    with pytest.raises(rkr_b200.RkrError):
        rkr_b200.build_thresholds_static(du.data_ptr(), 4, di.data_ptr(), 20000, 8, too_many, out.data_ptr())
