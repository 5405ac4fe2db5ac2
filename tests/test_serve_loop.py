"""The config-5 serving loop of bench.py, on the CPU with a stand-in server: the seeded trace (sizes,
k, arrival order), the order in which requests are submitted, and the latency/throughput summary."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
import bench  # noqa: E402


class FakeServer:
    """Stands in for rkr_b200.Server: records the requests in submission order and answers each at once."""
    log = []

    def __init__(self, index, method, max_batch_queries, n_workers, workspace_bytes):
        self.method = method
        self.n = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        pass

    def submit(self, q, ks):
        assert q.dtype == np.float32 and q.ndim == 2 and ks.shape == (q.shape[0],)
        FakeServer.log.append((self.method, q.shape[0], int(ks[0]), float(q[0, 0])))
        self.n += 1
        return self.n

    def wait(self, ticket, timeout=-1.0):
        return [], {"done": 1e-4, "start": 0.0}

    def counters(self):
        return {"batches": self.n, "requests": self.n, "queries": 0, "padded": 0, "busy_s": 0.0}


class FakeR:
    Server = FakeServer


def test_trace_is_seeded_and_submitted_in_arrival_order():
    item = np.random.default_rng(0).standard_normal((500, 8)).astype(np.float32)
    FakeServer.log = []
    arr, st, en, sz, cnt = bench.serve(FakeR, None, item, 8, 3, "QSRPNormalLP", 40, 20000.0)
    first = [c for c in FakeServer.log if c[1] == sz[0]]
    trace = FakeServer.log[-40:]
    FakeServer.log = []
    arr2, _, _, sz2, _ = bench.serve(FakeR, None, item, 8, 3, "QSRPNormalLP", 40, 20000.0)
    assert trace == FakeServer.log[-40:] and np.array_equal(sz, sz2) and first
    assert np.all(np.diff(arr) >= 0) and np.all(st >= arr - 1e-9) and np.all(en >= st)
    assert [c[1] for c in trace] == list(sz)
    assert all(1 <= n <= 256 and 10 <= k <= 200 for _, n, k, _ in trace)
    assert cnt["requests"] == 40


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
