"""bench.py's reference arm (--impl reference), on the CPU.

The arm times the reference's own QSRPNormalLP::Retrieval (oracle/_ref) on an index it builds on
the host without the engine library.  These tests run it end to end at the CPU-sized workload,
check that the engine's librkr_b200.so is never mapped into that process, and check the host
build's stand-in score rows against the reference's own build stages on a small case.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from checkers import Reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not Reference.available(), reason="oracle/_ref not built")

PROBE = r'''
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--config", "config1", "--steps", "2", "--warmup", "1",
            "--cpu-seconds", "0.4"]
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"engine_loaded": "librkr_b200" in maps, "torch_loaded": "torch" in sys.modules}))
'''


@needs_ref
def test_reference_arm_runs_without_the_engine():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 2, r.stdout
    line, probe = lines
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "queries/s"
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["cpu_model"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert not probe["engine_loaded"], "the reference arm mapped librkr_b200.so"
    assert not probe["torch_loaded"]


@needs_ref
def test_reference_arm_stage_outputs_match_the_reference_build(monkeypatch):
    """The host build's BLAS score rows stand in for the reference's sequential sums: the query-rank
    distribution and the thresholds agree with the reference's own build stages up to the last bit of
    a few scores (near-ties may move a user by one rank)."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setitem(bench.CONFIGS, "tiny", (600, 2500, 24, 48, 150, 10, 50, 10))
    rng = np.random.default_rng(5)
    user_raw = rng.standard_normal((600, 24)).astype(np.float32)
    item = rng.standard_normal((2500, 24)).astype(np.float32)
    parts, stages = bench.build_index_reference(user_raw, item, "tiny", 4)
    ref = Reference(4)
    user = ref.normalize(user_raw)
    assert np.array_equal(parts["user"].view(np.int32), user.view(np.int32))
    thr = ref.build_thresholds(user, item, parts["rank"])
    np.testing.assert_allclose(parts["thr"], thr, rtol=0, atol=1e-5)
    assert (np.diff(parts["thr"], axis=1) <= 0).all()
    si = ref.sample_item(2500, 150)
    accu = ref.query_rank_distribution(user, item, si)
    ranks = np.empty((600, 150), np.int32)
    # the stand-in's accu is not returned; recompute it the same way to compare with the reference's
    rows = user @ item.T
    s = rows[:, si]
    rows.sort(axis=1)
    for i in range(600):
        ranks[i] = 2500 - np.searchsorted(rows[i], s[i], side="right")
    mine = np.stack([np.cumsum(np.bincount(ranks[:, j], minlength=2501)) for j in range(150)])
    assert np.abs(mine - accu).max() <= 2
    assert set(stages) >= {"query_rank_distribution", "thresholds", "regression_fit", "svd"}


def test_bench_sequential_binary32_sum_is_the_reference_inner_product():
    """The bench's score-error report compares the tensor-core estimates with the reference's
    InnerProduct restated in numpy (seq_dot32); it equals the oracle's, bit for bit."""
    sys.path.insert(0, ROOT)
    import bench
    from checkers import Oracle
    orc = Oracle()
    rng = np.random.default_rng(8)
    a = rng.standard_normal((7, 150)).astype(np.float32)
    b = (rng.standard_normal((5, 150)) * 3).astype(np.float32)
    got = bench.seq_dot32(a, b)
    for i in range(7):
        for j in range(5):
            assert np.float32(orc.inner_product(a[i], b[j])).view(np.int32) == got[i, j].view(np.int32)
