"""The config-5 serving loop of bench.py, on the CPU with a stand-in index: the seeded trace (sizes,
k, arrival order) and the order of the calls, which QSRPNormalLP's carried per-user scores make part
of the answer, and the latency/throughput summary."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
import bench  # noqa: E402


class FakeIndex:
    def __init__(self):
        self.calls = []

    def retrieval(self, method, q, k):
        assert q.dtype == np.float32 and q.ndim == 2
        self.calls.append((method, q.shape[0], k, float(q[0, 0])))


def test_trace_is_seeded_and_answered_in_arrival_order():
    item = np.random.default_rng(0).standard_normal((500, 8)).astype(np.float32)
    a, b = FakeIndex(), FakeIndex()
    arr, st, en, sz = bench.serve(a, item, 8, 3, "QSRPNormalLP", 40, 20000.0)
    arr2, _, _, sz2 = bench.serve(b, item, 8, 3, "QSRPNormalLP", 40, 20000.0)
    assert a.calls == b.calls and np.array_equal(arr, arr2) and np.array_equal(sz, sz2)
    assert np.all(np.diff(arr) > 0) and np.all(st >= arr - 1e-9) and np.all(en >= st) and np.all(np.diff(st) >= 0)
    assert [c[1] for c in a.calls] == list(sz)
    assert all(1 <= n <= 256 and 10 <= k <= 200 for _, n, k, _ in a.calls)


def test_summary_counts_queueing():
    arr = np.array([0.0, 0.001, 0.002])
    st = np.array([0.0, 0.010, 0.020])
    en = np.array([0.010, 0.020, 0.030])
    sz = np.array([10, 20, 30])
    s = bench.serve_summary(arr, st, en, sz, 1000.0)
    assert s["requests"] == 3 and s["queries"] == 60
    assert abs(s["service_ms"]["mean"] - 10.0) < 1e-9
    assert abs(s["latency_ms"]["p50"] - 19.0) < 1e-9  # the second request waited 9 ms in the queue
    assert abs(s["throughput_req_per_s"] - 100.0) < 1e-6
