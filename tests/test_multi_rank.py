"""The replica form of a multi-GPU run (bench.py under torchrun) on the CPU: two `gloo` ranks on
127.0.0.1.  Each rank draws its own query batches (independent seeded streams), the job's time is
the slowest rank's (all-reduce MAX, every rank taking part), and the whole-job rate counts the units
of all ranks; a rank whose batches fail to match the others' shapes would show here first."""
import os
import socket
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, item, qrng = bench.make_data("config1", 0, rank)
        batch = item[qrng.choice(item.shape[0], size=16, replace=False)]
        got = [torch.zeros((16, item.shape[1])) for _ in range(world)]
        dist.all_gather(got, torch.from_numpy(batch))
        t = bench.max_over_ranks(0.5 + rank, dist, "cpu")
        rate = bench.job_rate(world, 100, t)
        dist.barrier()
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), batches=np.stack([g.numpy() for g in got]), t=t, rate=rate)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [np.load(os.path.join(tmp_path, f"r{i}.npz")) for i in range(world)]
    for x in r:
        assert float(x["t"]) == 1.5                      # the slowest rank's time, on every rank
        assert abs(float(x["rate"]) - 2 * 100 / 1.5) < 1e-9
    assert np.array_equal(r[0]["batches"], r[1]["batches"])   # the all-gather agrees on both ranks
    assert not np.array_equal(r[0]["batches"][0], r[0]["batches"][1])  # ranks draw different queries
