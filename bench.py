#!/usr/bin/env python
"""Benchmark of the reverse k-ranks query path on B200 (QSRPNormalLP, exact reference ranks).

Workload (default, --config config2): 480,189 users x 17,770 items, d = 150; users N(0, 1/150),
items N(0, 1/150) scaled per item by lognormal(0, 0.3); the index holds 512 sampled thresholds per
user (ranks chosen by the OptimalPart program over 150 sampled items, sample_topk = 100), one
NormalLinearRegressionLP model per user and the SVD transform (sigma 0.7).  A step is one batch of
1,000 query items drawn uniformly from the items, answered at k = 100.  Synthetic, seeded data
stands in for the reference's matrix-factorisation datasets (not available here).

value      queries/s with the queries and results resident in device memory (CUDA events on the
           launching stream, max over ranks);
e2e        queries/s through the public host API (rkr_retrieval), host->device copy of the queries
           and device->host copy of the results inside every timed step;
roofline   the dominant kernel's algorithmic throughput from live per-kernel event timing;
plain_fp32_gpu  the same batches through the engine's exact FP32 SIMT form (no tensor cores:
           exact register-tiled score tiles and refinement tiles), the baseline the metric names;
           vs_baseline = value / its value;
cpu_baseline  the reference's own QSRPNormalLP::Retrieval (oracle/_ref) on a bounded sample of
           the same queries, all host threads.
--impl reference times only that reference path and prints its line.  Its index is built on the
host without the engine library: the reference's own normalisation, sample-item draw, sample-rank
program, regression fit and SVD (oracle/_ref), with score rows from a BLAS product sorted per
user (numpy), standing in for the reference's ComputeScoreTableBatch rows.

Multi-GPU (torchrun): every rank holds a replica of the index and answers its own batch of
queries (weak scaling, no collective on the data path).
"""
import argparse
import contextlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "reverse-k-ranks_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "queries/sec and p50/p99 ms at exact ranks (k=100) vs plain FP32 GPU; index-build sec"

CONFIGS = {
    # name: n_user, n_item, dim, n_sample, n_sample_item, sample_topk, batch, topk
    "config2": (480189, 17770, 150, 512, 150, 100, 1000, 100),
    "config1": (1000, 5000, 30, 64, 150, 10, 100, 10),
    "config4": (1000990, 624961, 150, 512, 150, 100, 1000, 100),
    # the config-4 index serving a seeded Poisson stream of requests (serve())
    "config5": (1000990, 624961, 150, 512, 150, 100, 1000, 100),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


@contextlib.contextmanager
def quiet_stdout():
    """Silence C-level stdout (the reference prints progress lines) so ours stays one JSON line."""
    sys.stdout.flush()
    fd = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)
    try:
        yield
    finally:
        sys.stdout.flush()
        os.dup2(fd, 1)
        os.close(fd)
        os.close(dn)


def make_data(cfg, seed, rank_id):
    n_user, n_item, dim = CONFIGS[cfg][:3]
    rng = np.random.default_rng(seed)
    user = rng.standard_normal((n_user, dim), dtype=np.float32) * np.float32(1 / np.sqrt(dim))
    item = rng.standard_normal((n_item, dim), dtype=np.float32) * np.float32(1 / np.sqrt(dim))
    if cfg in ("config2", "config4", "config5"):
        item *= np.exp(rng.normal(0.0, 0.3, (n_item, 1))).astype(np.float32)
    qrng = np.random.default_rng(seed + 1000 + rank_id)
    return user, item, qrng


def max_over_ranks(x, dist, device):
    """x on this rank -> its maximum over all ranks (every rank takes part; the job's time is its
    slowest rank's)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, seconds):
    """Whole-job throughput of a replica run: every rank processes units_per_rank (weak scaling),
    timed by the slowest rank."""
    return world * units_per_rank / seconds


def build_index(R, user_raw, item, cfg, device):
    n_user, n_item, dim, n_sample, n_si, stopk = CONFIGS[cfg][:6]
    stages = {}
    t = time.perf_counter()
    user = R.normalize(user_raw)
    stages["normalize"] = time.perf_counter() - t
    t = time.perf_counter()
    ix = R.Index(user, item, device=device)
    stages["upload"] = time.perf_counter() - t
    t = time.perf_counter()
    si = R.sample_item(n_item, n_si)
    accu = ix.query_rank_distribution(si)
    stages["query_rank_distribution"] = time.perf_counter() - t
    t = time.perf_counter()
    kth, sid = R.sort_kth_rank(accu, stopk)
    rank, _ = R.find_optimal_sample_rank(n_user, n_item, n_sample, kth, accu[sid])
    stages["sample_rank"] = time.perf_counter() - t
    t = time.perf_counter()
    thr = ix.build_sample_search(rank)
    stages["thresholds"] = time.perf_counter() - t
    t = time.perf_counter()
    reg = ix.fit_regression()  # on the device, from the resident thresholds; loaded as the index's models
    stages["regression_fit"] = time.perf_counter() - t
    t = time.perf_counter()
    ti, su, cd = ix.svd_build(0.7)  # Gram matrix and projection on the device; made the index's
    stages["svd"] = time.perf_counter() - t
    parts = dict(user=user, rank=rank, thr=thr, reg=reg, ti=ti, su=su, cd=cd)
    return ix, parts, stages


def _score_blocks(user, item, n_thread, block, fn):
    """Calls fn(u0, rows) for consecutive blocks of users, rows = user[u0:u0+block] @ item.T (BLAS,
    float32), on n_thread host threads (numpy releases the GIL in the product and the sort)."""
    from concurrent.futures import ThreadPoolExecutor

    def one(u0):
        fn(u0, user[u0:u0 + block] @ item.T)

    with ThreadPoolExecutor(max(1, n_thread)) as ex:
        list(ex.map(one, range(0, user.shape[0], block)))


def build_index_reference(user_raw, item, cfg, n_thread):
    """The reference arm's index, built on the host without the engine library.

    The reference's own code (oracle/_ref) normalises the users (readData), draws the sampled items
    (SampleItem), picks the sample ranks (ComputeSortKthRank, FindOptimalSampleFast), fits the
    regression models (NormalLinearRegressionLP) and the SVD transform.  The score rows its build apps
    sort (ComputeScoreTableBatch, QueryRankByComputation) come from a float32 BLAS product sorted per
    user: the same index up to the last bit of a few scores, built in seconds instead of the
    reference's CPU build (about 15 minutes on 16 threads at config 2).  Returns the parts
    ReferenceTimer takes and the stage times."""
    from checkers import Reference
    n_user, n_item, dim, n_sample, n_si, stopk = CONFIGS[cfg][:6]
    ref = Reference(n_thread)
    stages = {}
    t = time.perf_counter()
    with quiet_stdout():
        user = ref.normalize(user_raw)
    stages["normalize"] = time.perf_counter() - t
    t = time.perf_counter()
    with quiet_stdout():
        si = ref.sample_item(n_item, n_si)
    ranks = np.empty((n_user, n_si), np.int32)

    def qrank(u0, rows):
        # rank of a sampled item = items scoring strictly above it (QueryRankByComputation.hpp)
        s = rows[:, si]
        rows.sort(axis=1)
        for i in range(rows.shape[0]):
            ranks[u0 + i] = n_item - np.searchsorted(rows[i], s[i], side="right")

    block = max(64, (256 << 20) // (4 * n_item))  # about 256 MB of score rows per thread
    _score_blocks(user, item, n_thread, block, qrank)
    accu = np.empty((n_si, n_item + 1), np.int32)
    for j in range(n_si):
        accu[j] = np.cumsum(np.bincount(ranks[:, j], minlength=n_item + 1))
    stages["query_rank_distribution"] = time.perf_counter() - t
    t = time.perf_counter()
    with quiet_stdout():
        rank, _ = ref.find_optimal_sample_rank(n_user, n_item, n_sample, si, accu, stopk)
    stages["sample_rank"] = time.perf_counter() - t
    t = time.perf_counter()
    thr = np.empty((n_user, n_sample), np.float32)
    desc = (n_item - 1 - rank).astype(np.int64)  # positions in an ascending row

    def thresholds(u0, rows):
        rows.sort(axis=1)
        thr[u0:u0 + rows.shape[0]] = rows[:, desc]

    _score_blocks(user, item, n_thread, block, thresholds)
    stages["thresholds"] = time.perf_counter() - t
    t = time.perf_counter()
    with quiet_stdout():
        reg = ref.fit_regression(thr, n_item, rank)
    stages["regression_fit"] = time.perf_counter() - t
    t = time.perf_counter()
    with quiet_stdout():
        ti, su, cd = ref.svd_build(user, item, 0.7)
    stages["svd"] = time.perf_counter() - t
    return dict(user=user, rank=rank, thr=thr, reg=reg, ti=ti, su=su, cd=cd), stages


def run_reference(args):
    """--impl reference: the reference's own QSRPNormalLP::Retrieval (oracle/_ref) on an index built
    without the engine (build_index_reference), each step a bounded sample of the step's batch on
    all host threads.  Touches no GPU."""
    n_user, n_item, dim, n_sample, n_si, stopk, batch, topk = CONFIGS[args.config]
    if args.batch:
        batch = args.batch
    if args.config == "config5":
        print(json.dumps({"impl": "reference", "unavailable": "config5 is a serving loop of the engine; the "
                          "reference arm is timed on config2/config4 batches"}))
        return
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference "
                          "sources at build time)"}))
        return
    n_thread = os.cpu_count() or 1
    log(f"[bench-ref] generating {args.config} data")
    user_raw, item, qrng = make_data(args.config, args.seed, 0)
    t0 = time.perf_counter()
    parts, stages = build_index_reference(user_raw, item, args.config, n_thread)
    build_sec = time.perf_counter() - t0
    log(f"[bench-ref] index built on the host in {build_sec:.1f}s: " +
        ", ".join(f"{k} {v:.2f}s" for k, v in stages.items()))
    timer = ReferenceTimer(parts, item, n_thread)
    runs = []
    for s in range(args.warmup + args.steps):
        q = item[qrng.choice(n_item, size=batch, replace=False)].copy()
        n, secs, _ = timer.run(q, topk, args.cpu_seconds / 4)
        if s >= args.warmup:
            runs.append((n, secs))
    timer.close()
    secs = sum(r[1] for r in runs)
    nqs = sum(r[0] for r in runs)
    v = nqs / secs
    model = cpu_model()
    sample = (f"the first {runs[-1][0]} of each step's {batch} queries through the reference's "
              f"QSRPNormalLP::Retrieval (oracle/_ref, the reference's unmodified headers), {n_thread} OpenMP "
              f"threads on {model}")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "queries/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(runs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded numpy N(0,1/150) users, lognormal-scaled N(0,1/150) items, queries drawn "
                    "from the items; index built on the host without the engine (reference code + BLAS rows)",
            "config": {"workload": f"{args.config}: {n_user} users x {n_item} items, d={dim}, {n_sample} sampled "
                                   f"thresholds/user + NormalLinearRegressionLP + SVD, QSRPNormalLP, "
                                   f"{batch} queries/step, k={topk}",
                       "sample_queries_per_step": int(round(nqs / len(runs)))},
            "build_sec_host": build_sec, "build_stages_sec": {k: round(v_, 3) for k, v_ in stages.items()},
            "cpu_baseline": {"value": v, "unit": "queries/s", "cores": n_thread, "cpu_model": model,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


class Clocks:
    """SM clock and throttle reasons while the timed region runs: one `nvidia-smi -lms 200` process
    started before warm-up and stopped after the timed steps; only samples inside the timed
    window (plus a margin) are summarised."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.window = None

    def __enter__(self):
        self.t0 = time.perf_counter()
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.lines = []
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.reader.join(timeout=5)
            self.samples = [(t, [x.strip() for x in l.split(",")]) for t, l in self.lines if l]

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def summary(self):
        w = self.window
        samples = [s for t, s in self.samples if w is None or w[0] - 0.3 <= t <= w[1] + 0.3]
        if not samples:
            samples = [s for _, s in self.samples[-3:]]
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples for i in range(4) if len(s) > 3 + i and
                          s[3 + i].lower() in ("active", "1")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(samples)}


def kernel_model(name, cfg, nq, stats, method):
    """Algorithmic (dot_flops, bytes, tensor_ops) per launch of the query kernels, from the workload's
    sizes.

    dot_flops counts the exact dot products' binary32 multiplies and adds as separate operations (2 per
    coordinate and pair).  bytes is what the kernel must move through HBM at the least: for the pair
    scores (the bound rounds' stream over the resident index) one pass over every user's vector at
    2 bytes a coordinate, its 28-byte regression record (QSRPNormalLP) and its S sampled thresholds,
    U * (2 d + 28 + 4 S) per batch, whatever the kernel itself stores per pair.  tensor_ops counts the
    tensor-core operations the kernel issues: ten int8 digit products per coordinate (K padded to 32
    per part)."""
    n_user, n_item, dim, n_sample = CONFIGS[cfg][:4]
    pairs = float(n_user) * nq
    r32 = lambda x: (x + 31) // 32 * 32
    if name == "qsrp_scores_tc":
        qsrp = method == "QSRPNormalLP"
        cd = stats["check_dim"] if qsrp else dim
        kp = r32(cd) + (r32(dim - cd) if dim > cd else 0)
        per_user = 2.0 * dim + (28.0 if qsrp else 0.0) + 4.0 * n_sample
        return 2.0 * pairs * dim, n_user * per_user + nq * 4.0 * dim, 10 * 2.0 * pairs * kp
    if name == "refine_tc":
        # per (candidate, item) pair in the norm cut-off; the items read once at the least
        n = stats["n_compute_item"]
        cd = stats["check_dim"] if method != "US" else dim
        kp = r32(cd) + (r32(dim - cd) if dim > cd else 0)
        return 2.0 * n * dim, 2.0 * dim * n_item, 10 * 2.0 * n * kp
    return 0.0, 0.0, 0.0


# DRAM traffic of the pair-scores kernel from one ncu capture at a 200-query batch of the config-2
# workload (dram__bytes_read.sum, dram__bytes_write.sum): the reads are the resident index (the
# users' digit tiles, threshold summaries and level tables), streamed once per launch whatever its
# queries; the writes are the two state bytes per (query, user) pair.  A launch's traffic is the
# read figure plus the write figure per pair times its pairs.
NCU_TRAFFIC = {("qsrp_scores_tc", "QSRPNormalLP"): (563.217e6, 170.901e6 / (200 * 480189.0))}

# Nominal dense tensor-core peaks of one B200 (T ops/s), for the tensor_ops figures.
TENSOR_PEAK_NOMINAL = {"qsrp_scores_tc": ("int8", 4500.0), "refine_tc": ("int8", 4500.0)}


def seq_dot32(a, b):
    """The reference's InnerProduct for every row pair: a sequential binary32 sum, one rounding per
    product and per addition (a [n][d], b [m][d] float32 -> [n][m])."""
    acc = np.zeros((a.shape[0], b.shape[0]), np.float32)
    for j in range(a.shape[1]):
        acc = acc + np.outer(a[:, j], b[:, j]).astype(np.float32)
    return acc


def score_error_report(ix, parts, item_queries, method, user_stride=24):
    """The tensor-core pair scores against the reference's binary32 scores and against FP64, on a
    sample of pairs (every user_stride-th user x the given queries): the largest error, and the
    largest ratio of the error to the bound the kernel holds (which must stay below 1)."""
    est = ix.score_estimates(method, item_queries)
    users = np.arange(0, est.shape[1], user_stride)
    e = est[:, users, 0].T.astype(np.float64)
    bound = est[:, users, 1].T.astype(np.float64)
    q = item_queries.astype(np.float32)
    if method == "QSRPNormalLP":
        ti, cd = parts["ti"], parts["cd"]
        qt = seq_dot32(q, ti)                        # SVD::TransferQuery, one sequential sum per coordinate
        u = parts["su"][users]
        ref = (seq_dot32(u[:, :cd], qt[:, :cd]) + seq_dot32(u[:, cd:], qt[:, cd:])).astype(np.float32)
    else:
        qt = q
        u = parts["user"][users]
        ref = seq_dot32(u, qt)
    fp64 = u.astype(np.float64) @ qt.astype(np.float64).T
    ok = np.isfinite(e)
    err64 = np.abs(e - fp64)[ok]
    err32 = np.abs(e - ref.astype(np.float64))[ok]
    return {"pairs": int(ok.sum()), "estimate": "int8 four-digit tensor-core products, int32 accumulation",
            "max_abs_err_vs_fp64": float(err64.max()) if err64.size else None,
            "mean_abs_err_vs_fp64": float(err64.mean()) if err64.size else None,
            "max_abs_err_vs_reference_binary32": float(err32.max()) if err32.size else None,
            "max_err_over_bound": float((err32 / bound[ok]).max()) if err32.size else None,
            "reference_binary32_max_abs_err_vs_fp64": float(np.abs(ref.astype(np.float64) - fp64).max())}


def cpu_model():
    """The host CPU's model name (first 'model name' line of /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ReferenceTimer:
    """The reference's QSRPNormalLP::Retrieval (oracle/_ref) held open on the same index; each run
    times a bounded sample of queries with all host threads."""

    def __init__(self, parts, item, n_thread, fast=False):
        from checkers import REF_FAST_SO, REF_SO, ReferenceQsrp
        self.n_thread = n_thread
        with quiet_stdout():
            self.ref = ReferenceQsrp(parts["user"], parts["su"], parts["ti"], item, parts["cd"], parts["rank"],
                                     parts["thr"], parts["rank"], parts["reg"], n_thread,
                                     so=REF_FAST_SO if fast else REF_SO)
        self.per_q = None

    def run(self, queries, topk, budget_s):
        """Times queries[:4] (calibration), then queries[:n]; returns n, the seconds of the second run
        and its results (the reference's state carries over from the first run, as in one index)."""
        with quiet_stdout():
            if self.per_q is None:
                _, _, t = self.ref.run(queries[:4], topk)
                self.per_q = max(t / 4, 1e-6)
            n = int(min(len(queries), max(8, budget_s / self.per_q)))
            res, _, secs = self.ref.run(queries[:n], topk)
        self.per_q = secs / n
        return n, secs, res

    def close(self):
        self.ref.close()


def reference_available():
    from checkers import Reference
    return Reference.available()


def serve(R, ix, item, dim, seed, method, n_req, rate, max_batch=1024, n_workers=2, workspace_bytes=0):
    """A serving run over a seeded Poisson arrival trace against the persistent server (rkr_server_*):
    each request holds 1-256 query items (uniform), drawn from the items or out-of-set N(0, 1/dim)
    vectors with equal odds, and one k ~ U[10, 200] for its items.  A submitter thread offers each
    request at its arrival time (open loop); the server batches whatever is queued (continuous
    batching, two batches in flight, graph replay) and answers each request as it would alone.
    Returns per-request arrival, start and end times (seconds from the trace's start), sizes and the
    server's counters."""
    rng = np.random.default_rng(seed + 5000)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    sizes = rng.integers(1, 257, n_req)
    ks = rng.integers(10, 201, n_req)
    from_items = rng.random(n_req) < 0.5
    reqs = []
    for i in range(n_req):
        if from_items[i]:
            q = item[rng.choice(item.shape[0], size=int(sizes[i]), replace=False)].copy()
        else:
            q = (rng.standard_normal((int(sizes[i]), dim)) / np.sqrt(dim)).astype(np.float32)
        reqs.append((q, np.full(int(sizes[i]), int(ks[i]), np.int32)))
    start = np.zeros(n_req)
    end = np.zeros(n_req)
    tickets = [None] * n_req
    submitted = threading.Semaphore(0)
    with R.Server(ix, method=method, max_batch_queries=max_batch, n_workers=n_workers,
                  workspace_bytes=workspace_bytes) as srv:
        # warm-up: every batch size the trace can produce runs once eagerly and once captured (the
        # server pads a batch to the next power of two; requests hold at most 256 items)
        for nb in (16, 32, 64, 128, 256, 512, 1024):
            if nb > max_batch:
                break
            for _ in range(2):
                w, left = [], nb
                while left > 0:
                    n = min(left, 256)
                    w.append(srv.submit(item[:n], np.full(n, 200 if n > 1 else 10, np.int32)))
                    left -= n
                for t in w:
                    srv.wait(t, timeout=600.0)
        c0 = srv.counters()
        t0 = time.perf_counter()

        def submitter():
            for i in range(n_req):
                now = time.perf_counter() - t0
                if now < arrivals[i]:
                    time.sleep(arrivals[i] - now)
                tickets[i] = (time.perf_counter() - t0, srv.submit(*reqs[i]))
                submitted.release()

        th = threading.Thread(target=submitter)
        th.start()
        for i in range(n_req):
            submitted.acquire()
            t_sub, tk = tickets[i]
            _, lat = srv.wait(tk, timeout=600.0)
            start[i] = t_sub + lat["start"]
            end[i] = t_sub + lat["done"]
            arrivals[i] = t_sub  # the offered time as actually submitted
        th.join()
        c1 = srv.counters()
    counters = {k: c1[k] - c0[k] for k in c1}
    return arrivals, start, end, sizes, counters


def serve_summary(arrivals, start, end, sizes, rate):
    lat = (end - arrivals) * 1e3
    svc = (end - start) * 1e3
    span = end.max() - arrivals[0]
    return {"offered_req_per_s": rate, "requests": int(len(sizes)), "queries": int(sizes.sum()),
            "throughput_req_per_s": len(sizes) / span, "throughput_queries_per_s": float(sizes.sum()) / span,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "service_ms": {"p50": float(np.percentile(svc, 50)), "p99": float(np.percentile(svc, 99)),
                           "mean": float(svc.mean())}}


def run_sharded(args, R, user_raw, item, qrng, dist, world, rank_id, local, batch, topk):
    """User shards (rkr_index_set_shard): rank r builds and holds its user range, the selection counts
    are summed over the ranks through NCCL on the engine's stream (rkr_b200.shard.TorchExchange), and
    every query's parts are gathered and merged on every rank.  Every rank draws the same queries.  The
    timed step is one batch end to end: host queries in, each rank's shard query, the gather of the
    parts and the merge (the whole answer on every rank)."""
    import socket
    import torch
    import torch.distributed as tdist
    from rkr_b200.shard import TorchExchange, shard_users
    own_group = dist is None
    if own_group:  # one rank: a one-member NCCL group, so that the exchange still runs through NCCL
        import datetime
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        store = tdist.TCPStore("127.0.0.1", port, 1, True, timeout=datetime.timedelta(seconds=60))
        tdist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=120))
    n_user, n_item, dim, n_sample, n_si, stopk = CONFIGS[args.config][:6]
    start, end = shard_users(n_user, world, rank_id)
    t0 = time.perf_counter()
    user_all = R.normalize(user_raw)
    ix = R.Index(user_all[start:end], item, device=local)
    ex = TorchExchange(None, torch.device("cuda", local))
    ix.set_shard(rank_id, world, start, n_user, (ex.fn, None))
    si = R.sample_item(n_item, n_si)
    accu = ix.query_rank_distribution(si)  # every shard's users (summed through the exchange)
    kth, sid = R.sort_kth_rank(accu, stopk)
    rank, _ = R.find_optimal_sample_rank(n_user, n_item, n_sample, kth, accu[sid])
    ix.build_sample_search(rank, return_thresholds=False)
    ix.fit_regression(records=False)
    ti, su, cd = R.svd_build(user_all, 0.7)  # the same transform on every rank (host, all users)
    ix.load_svd(cd, ti, su[start:end])
    torch.cuda.synchronize()
    build_sec = time.perf_counter() - t0
    ks = np.full(batch, topk, np.int32)
    batches = [item[qrng.choice(n_item, size=batch, replace=False)].copy() for _ in range(args.warmup + args.steps)]

    def step(q):
        part, front, st = ix.shard_query(args.method, q, ks, stats=True)
        if dist is None:
            return R.shard_merge(ks, [part], [front], [st])
        got = [None] * world
        dist.all_gather_object(got, (part, front, st))
        return R.shard_merge(ks, [g[0] for g in got], [g[1] for g in got], [g[2] for g in got])

    stream = torch.cuda.current_stream()
    with Clocks(local) as clk:
        time.sleep(0.5)
        for s in range(args.warmup):
            step(batches[s])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        wall0 = time.perf_counter()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(args.steps):
            out, mst = step(batches[args.warmup + s])
        e1.record(stream)
        torch.cuda.synchronize()
        clk.mark(wall0, time.perf_counter())
    total_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    value = batch * args.steps / (total_ms / 1e3)  # the same queries on every rank: the job answers them once
    if rank_id == 0:
        line = {"metric": "queries/sec at exact ranks over user shards (k=%d)" % topk, "value": value,
                "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy), the workload's shapes",
                "config": {"workload": f"{args.config}: {n_user} users x {n_item} items, d={dim}, {n_sample} sampled "
                                       f"thresholds/user, {args.method}, {batch} queries/step, k={topk}; user shards",
                           "shard_users": [end - start], "parallelism": f"user shards x{world}",
                           "l2": "inputs larger than L2 (resident index >= 1.6 GB)" if args.config != "config1"
                           else "small"},
                "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": batch * dim * 4,
                        "d2h_bytes_per_step": int(out.nbytes)},
                "build_sec": build_sec, "clocks": clk.summary()}
        print(json.dumps(line))
    ix.close()
    if own_group:
        tdist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="config2", choices=sorted(CONFIGS))
    ap.add_argument("--method", default="QSRPNormalLP", choices=["QSRPNormalLP", "QS", "US"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--single-queries", type=int, default=100)
    ap.add_argument("--batch", type=int, default=0, help="queries per step (default: the workload's)")
    ap.add_argument("--shard-users", action="store_true",
                    help="user shards instead of replicas: rank r holds users [r U/N, (r+1) U/N), every rank "
                         "answers the same queries for its users, the parts are merged (strong scaling)")
    ap.add_argument("--n-user", type=int, default=0,
                    help="users of the workload (default: the configuration's); smaller for profiler captures")
    ap.add_argument("--serve-requests", type=int, default=200, help="config5: requests per trace")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="config5: offered requests/s")
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="skip timing the plain FP32 GPU form")
    args = ap.parse_args()
    if args.n_user:
        CONFIGS[args.config] = (args.n_user,) + CONFIGS[args.config][1:]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank_id = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # rank 0 alone times the reference's CPU path; other ranks exit without work
        if rank_id == 0:
            run_reference(args)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    n_user, n_item, dim, n_sample, n_si, stopk, batch, topk = CONFIGS[args.config]
    if args.batch:
        batch = args.batch
    elif args.method == "US":
        batch = 100  # US answers exactly 100 queries per call when S <= 1000 (US.hpp:117-131)
    n_thread = os.cpu_count() or 1

    import rkr_b200 as R
    log(f"[bench] rank {rank_id}/{world}: generating {args.config} data")
    user_raw, item, qrng = make_data(args.config, args.seed, 0 if args.shard_users else rank_id)
    if args.shard_users:
        run_sharded(args, R, user_raw, item, qrng, dist, world, rank_id, local, batch, topk)
        if dist:
            dist.destroy_process_group()
        return
    t0 = time.perf_counter()
    ix, parts, stages = build_index(R, user_raw, item, args.config, local)
    torch.cuda.synchronize()
    build_sec = time.perf_counter() - t0
    log(f"[bench] index built in {build_sec:.2f}s: " + ", ".join(f"{k} {v:.2f}s" for k, v in stages.items()))

    def draw_batch():
        return item[qrng.choice(n_item, size=batch, replace=False)].copy()

    if args.config == "config5":
        if rank_id != 0:
            ix.close()
            if dist:
                dist.destroy_process_group()
            return
        with Clocks(local) as clk:
            t_a = time.perf_counter()
            arr, st_, en, sz, cnt = serve(R, ix, item, dim, args.seed, args.method, args.serve_requests,
                                          args.serve_rate)
            offered = serve_summary(arr, st_, en, sz, args.serve_rate)
            offered["server"] = cnt
            # the same kind of trace at 70% of the throughput the first trace sustained
            cap = offered["throughput_req_per_s"]
            arr, st_, en, sz, cnt = serve(R, ix, item, dim, args.seed + 1, args.method, args.serve_requests,
                                          0.7 * cap)
            sustained = serve_summary(arr, st_, en, sz, 0.7 * cap)
            sustained["server"] = cnt
            clk.mark(t_a, time.perf_counter())
        line = {"metric": "serving: request latency p50/p99 (ms) and throughput under Poisson arrivals",
                "value": offered["latency_ms"]["p99"], "unit": "ms (p99 request latency at the offered rate)",
                "higher_is_better": False, "n_gpus": 1, "dtype": "f32",
                "data": "synthetic: seeded numpy N(0,1/150) users, lognormal-scaled N(0,1/150) items; requests of "
                        "1-256 queries, half drawn from the items, half out-of-set N(0,1/150); k ~ U[10,200]",
                "config": {"workload": f"config5: the config4 index ({n_user} users x {n_item} items, d={dim}, "
                                       f"{n_sample} sampled thresholds/user + NormalLinearRegressionLP + SVD), "
                                       f"{args.method}, Poisson arrivals, persistent server: continuous "
                                       f"batching of up to 1024 query items, 2 batches in flight, phase-1 graph "
                                       f"replay, each request answered as alone", "seed": args.seed},
                "offered": offered, "at_70pct_capacity": sustained, "capacity_req_per_s": cap,
                "build_sec": build_sec, "hbm_index_bytes": ix.size_bytes(), "clocks": clk.summary()}
        print(json.dumps(line))
        ix.close()
        return

    # ---- device-resident timing -------------------------------------------------------------------
    stream = torch.cuda.current_stream()
    rec_bytes = R.USER_RANK.itemsize
    d_out = torch.empty(batch * topk * rec_bytes, dtype=torch.uint8, device="cuda")
    d_stats = torch.empty(batch * R.QUERY_STATS.itemsize, dtype=torch.uint8, device="cuda")
    batches = [torch.from_numpy(draw_batch()).cuda() for _ in range(args.warmup + args.steps)]

    def run_step(dq):
        return ix.retrieval_device(args.method, dq.data_ptr(), batch, topk, d_out.data_ptr(), d_stats.data_ptr(),
                                   stream=stream.cuda_stream)

    with Clocks(local) as clk:
        time.sleep(0.5)  # the sampler's first nvidia-smi call lands before the timed region
        for s in range(args.warmup):
            run_step(batches[s])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        step_ms = []
        wall0 = time.perf_counter()
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record(stream)
        for s in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run_step(batches[args.warmup + s])
            e1.record(stream)
            step_ms.append((e0, e1))
        t_all1.record(stream)
        torch.cuda.synchronize()
        clk.mark(wall0, time.perf_counter())
    total_ms = t_all0.elapsed_time(t_all1)
    step_ms = [a.elapsed_time(b) for a, b in step_ms]
    log("[bench] step ms: " + " ".join(f"{v:.2f}" for v in step_ms))
    total_ms = max_over_ranks(total_ms, dist, "cuda")
    value = job_rate(world, batch * args.steps, total_ms / 1e3)

    # ---- the plain FP32 GPU form on the same batches ---------------------------------------------------
    # A second index over the same data with the tensor-core paths off: exact register-tiled FP32
    # score tiles and refinement tiles (the results are the same; only the arithmetic path differs).
    plain = None
    if args.plain:
        os.environ["RKR_SCORES_TC"] = "0"
        os.environ["RKR_REFINE_TC"] = "0"
        try:
            ixp = R.Index(parts["user"], item, device=local)
        finally:
            os.environ.pop("RKR_SCORES_TC")
            os.environ.pop("RKR_REFINE_TC")
        ixp.load_sample_search(parts["rank"], parts["thr"])
        ixp.load_svd(parts["cd"], parts["ti"], parts["su"])
        ixp.load_regression(parts["rank"], parts["reg"])
        d_out_p = torch.empty_like(d_out)

        def run_plain(dq):
            return ixp.retrieval_device(args.method, dq.data_ptr(), batch, topk, d_out_p.data_ptr(), 0,
                                        stream=stream.cuda_stream)

        for s in range(args.warmup):
            run_plain(batches[s])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for s in range(args.steps):
            run_plain(batches[args.warmup + s])
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(p0.elapsed_time(p1), dist, "cuda")
        # the same queries answered by both forms (both started from the same carried state) agree
        ix.reset_state()
        ixp.reset_state()
        run_step(batches[0])
        run_plain(batches[0])
        torch.cuda.synchronize()
        same_plain = bool(torch.equal(d_out, d_out_p))
        ixp.close()
        plain = {"value": job_rate(world, batch * args.steps, plain_ms / 1e3), "unit": "queries/s",
                 "ms_per_step": plain_ms / args.steps,
                 "form": "exact FP32 SIMT tiles for the pair scores and the refinement (RKR_SCORES_TC=0 "
                         "RKR_REFINE_TC=0), same pipeline otherwise",
                 "results_identical": same_plain}

    # ---- per-kernel profile of one more step (outside the timed region) ---------------------------------
    ix.profile(True)
    run_step(batches[0])
    torch.cuda.synchronize()
    prof = ix.profile_read()
    ix.profile(False)
    is_counter = lambda k: k.endswith("_pairs") or k.endswith("_queries") or k.endswith("_rows")
    counters = {k: int(v[1]) for k, v in prof.items() if is_counter(k)}
    prof = {k: v for k, v in prof.items() if not is_counter(k)}
    st = np.frombuffer(d_stats.cpu().numpy().tobytes(), dtype=R.QUERY_STATS)
    model_stats = {"check_dim": parts["cd"], "n_compute_item": float(st["n_compute_item"].sum())}
    launches_per_step = sum(c for _, c in prof.values())
    stats_mean = {f: float(st[f].mean()) for f in R.QUERY_STATS.names}
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_n) = dom
    ops, nbytes, tops = kernel_model(dom_name, args.config, batch, model_stats, args.method)
    avg_s = dom_ms / 1e3 / max(dom_n, 1)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    ncu_t = NCU_TRAFFIC.get((dom_name, args.method))
    launches = max(1, -(-batch // 1024))  # the scores kernel takes up to 1,024 queries per launch
    traffic = (ncu_t[0] + ncu_t[1] * CONFIGS[args.config][0] * batch / launches
               if ncu_t is not None and args.config == "config2" else None)
    roofline = {"kernel": dom_name, "bound": "hbm", "achieved": nbytes / avg_s / 1e9, "peak": hbm_peak,
                "unit": "GB/s", "frac": (nbytes / avg_s / 1e9) / hbm_peak,
                "peak_source": "MEASURED_PEAKS.json (of measured)" if peaks else "fallback",
                "algorithmic_bytes": nbytes, "traffic": traffic,
                "traffic_over_algorithmic": traffic / nbytes if traffic and nbytes else None,
                "avg_launch_ms": avg_s * 1e3,
                "share_of_step": dom_ms / max(sum(v[0] for v in prof.values()), 1e-9),
                "dot_tflops_fp32_equivalent": ops / avg_s / 1e12}
    if dom_name in TENSOR_PEAK_NOMINAL:
        kind, peak = TENSOR_PEAK_NOMINAL[dom_name]
        roofline["tensor"] = {"kind": kind, "achieved_tops": tops / avg_s / 1e12, "peak_tops_nominal": peak,
                              "frac": tops / avg_s / 1e12 / peak}
    roofline.update({
                "kernels_ms_per_step": {k: round(v[0], 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
                "counters_per_step": counters})

    # ---- the tensor-core screen's estimates against the reference's scores and FP64 -------------------------
    score_err = None
    if args.method != "US":
        score_err = score_error_report(ix, parts, batches[0].cpu().numpy()[:32], args.method)
        ix.reset_state()

    # ---- latency ------------------------------------------------------------------------------------------
    single = []
    q1 = batches[0]
    # US answers exactly 100 queries per call when S <= 1000 (US.hpp:117-131): no single-query latency
    n_single = 0 if args.method == "US" else args.single_queries
    for i in range(n_single):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ix.retrieval_device(args.method, q1[i % batch:].data_ptr(), 1, topk, d_out.data_ptr(), 0,
                            stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        single.append(e0.elapsed_time(e1))

    # ---- end to end through the host API -----------------------------------------------------------------
    pinned = [torch.from_numpy(draw_batch()).pin_memory() for _ in range(args.steps)]
    # the results land in one pinned host buffer, reused by every call (as a C-ABI caller passes its own)
    res_host = torch.empty(batch * topk * R.USER_RANK.itemsize, dtype=torch.uint8).pin_memory()
    res_buf = res_host.numpy().view(R.USER_RANK).reshape(batch, topk)
    for s in range(min(2, args.warmup)):
        ix.retrieval(args.method, pinned[s % len(pinned)].numpy(), topk, out=res_buf)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t = time.perf_counter()
    for s in range(args.steps):
        res = ix.retrieval(args.method, pinned[s].numpy(), topk, out=res_buf)
    e2e_s = time.perf_counter() - t
    e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    e2e = {"value": job_rate(world, batch * args.steps, e2e_s), "unit": "queries/s",
           "h2d_bytes_per_step": batch * dim * 4, "d2h_bytes_per_step": batch * topk * rec_bytes}

    cpu = None
    if rank_id == 0 and world == 1 and args.method == "QSRPNormalLP" and reference_available():
        timer = ReferenceTimer(parts, item, n_thread)
        qs = batches[0].cpu().numpy()
        n, secs, ref_res = timer.run(qs, topk, args.cpu_seconds)
        timer.close()
        # the same calls through the engine from a fresh carried state: results must be identical
        ix.reset_state()
        ix.retrieval(args.method, qs[:4], topk)
        got = ix.retrieval(args.method, qs[:n], topk)
        flat = lambda x: np.ascontiguousarray(x).view(np.int32).reshape(-1)
        same = got.shape == ref_res.shape and np.array_equal(flat(got), flat(ref_res))
        cpu = {"value": n / secs, "unit": "queries/s", "cores": n_thread, "cpu_model": cpu_model(), "kind": "reference",
               "sample": f"{n} of the step's {batch} queries through the reference's QSRPNormalLP::Retrieval "
                         f"(oracle/_ref, the reference's unmodified headers) on the same index, {n_thread} threads",
               "results_identical_to_engine": bool(same)}
        # the reference's own CPU build stages (score rows, per-user sort, thresholds; the query-rank
        # distribution) on a subset of the users, extrapolated linearly to all of them as bstb does
        # (BuildScoreTableBatch.cpp:56-64, 143-144)
        from checkers import Reference
        refb = Reference(n_thread)
        n_sub = int(min(n_user, max(256, 2000 * 150 * 17770 // max(1, dim * n_item))))
        sub = parts["user"][:n_sub]
        t = time.perf_counter()
        with quiet_stdout():
            refb.query_rank_distribution(sub, item, R.sample_item(n_item, n_si))
        t_qd = time.perf_counter() - t
        t = time.perf_counter()
        with quiet_stdout():
            refb.build_thresholds(sub, item, parts["rank"])
        t_thr = time.perf_counter() - t
        cpu["build_extrapolated_sec"] = {"query_rank_distribution": t_qd * n_user / n_sub,
                                         "thresholds": t_thr * n_user / n_sub, "users_timed": n_sub,
                                         "threads": n_thread}
        from checkers import REF_FAST_SO
        if os.path.exists(REF_FAST_SO):
            # the same path under the reference's Release flags (-Ofast), timing only: its sums may
            # reassociate, so its results are not compared
            timer = ReferenceTimer(parts, item, n_thread, fast=True)
            nf, secs_f, _ = timer.run(qs, topk, args.cpu_seconds / 2)
            timer.close()
            cpu["ofast"] = {"value": nf / secs_f, "unit": "queries/s", "cores": n_thread,
                            "sample": f"{nf} of the same queries, oracle/_ref/librkr_ref_fast.so (-Ofast)"}

    if rank_id == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": (value / plain["value"]) if plain else None,
            "vs_baseline_basis": "value / plain_fp32_gpu.value (the plain FP32 GPU form the metric names, "
                                 "timed on the same batches in the same run; no published number exists)",
            "dtype": "f32",
            "data": "synthetic: seeded numpy N(0,1/150) users, lognormal-scaled N(0,1/150) items, queries drawn "
                    "from the items",
            "config": {"workload": f"{args.config}: {n_user} users x {n_item} items, d={dim}, {n_sample} sampled "
                                   f"thresholds/user + NormalLinearRegressionLP + SVD, {args.method}, "
                                   f"{batch} queries/step, k={topk}",
                       "batch_per_gpu": batch, "topk": topk, "method": args.method,
                       "l2": "inputs larger than L2 (resident index >= 1.6 GB)",
                       "parallelism": f"replica x{world} (queries split across GPUs)"},
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "single_query_p50_ms": float(np.percentile(single, 50)) if single else None,
            "single_query_p99_ms": float(np.percentile(single, 99)) if single else None,
            "build_sec": build_sec, "build_stages_sec": {k: round(v, 3) for k, v in stages.items()},
            "hbm_index_bytes": ix.size_bytes(), "e2e": e2e, "gpu_launches": int(launches_per_step * args.steps), "roofline": roofline,
            "plain_fp32_gpu": plain, "score_error": score_err, "cpu_baseline": cpu, "clocks": clk.summary(), "query_stats_mean": stats_mean,
        }
        print(json.dumps(line))
    ix.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
