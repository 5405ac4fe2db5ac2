"""User shards over torch.distributed: one process per GPU, each holding a contiguous range of users.

``TorchExchange`` is the count exchange a shard's queries need (``Index.set_shard``): an in-place SUM
all-reduce of the small per-query count arrays the engine selects from.  With device memory it runs
on the engine's CUDA stream (NCCL, no host synchronisation); with host memory (stream 0) it runs on
the CPU (gloo).  ``shard_users`` gives each rank its user range, and ``ShardedIndex`` builds one
rank's shard and answers whole queries (every rank's part gathered on every rank and merged by
``shard_merge``).  The reference holds every user in one process; its one global step is
PruneCandidateByBound (src/include/alg/RankBoundRefinement/PruneCandidateByBound.hpp:19-179).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from . import EXCHANGE_FN, QUERY_STATS, USER_RANK, Index, exchange_callback, shard_merge


def shard_users(n_user, n_shards, shard):
    """Users [start, end) of shard `shard`: contiguous, as even as possible, in shard order."""
    base, extra = divmod(int(n_user), int(n_shards))
    start = shard * base + min(shard, extra)
    return start, start + base + (1 if shard < extra else 0)


class _DeviceInts:
    """A device int32 array by address, for torch.as_tensor (CUDA array interface, no copy)."""

    def __init__(self, address, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (address, False),
                                         "version": 3, "strides": None, "stream": None}


class TorchExchange:
    """rkr_exchange_fn over a torch.distributed process group (every rank one shard)."""

    def __init__(self, group=None, device=None):
        self.group = group
        self.device = torch.device(device) if device is not None else None
        self.fn = exchange_callback(self)  # EXCHANGE_FN; kept alive with this object
        self._views = {}  # (address, n, stream) -> (stream object, tensor view): the engine reuses its buffers

    def __call__(self, address, n, stream):
        if n <= 0:
            return
        if stream:
            # device counts, ordered on the engine's stream: NCCL waits for the work queued there and
            # the stream waits for the sum
            key = (address, n, stream)
            view = self._views.get(key)
            if view is None:
                if len(self._views) > 256:
                    self._views.clear()
                s = torch.cuda.ExternalStream(stream, device=self.device)
                view = (s, torch.as_tensor(_DeviceInts(address, n), device=self.device))
                self._views[key] = view
            with torch.cuda.stream(view[0]):
                dist.all_reduce(view[1], op=dist.ReduceOp.SUM, group=self.group)
        else:
            a = np.ctypeslib.as_array((C.c_int32 * n).from_address(address))
            t = torch.from_numpy(a)
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)


class ShardedIndex:
    """One rank's shard of an index over `user` (all users, the same on every rank; this rank
    uploads its range only) and `item`, and whole-query answers through the merge."""

    def __init__(self, user, item, device=0, group=None):
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.group = group
        self.n_user_total = int(user.shape[0])
        self.start, self.end = shard_users(self.n_user_total, self.world, self.rank)
        self.index = Index(user[self.start:self.end], item, device)
        dev = torch.device("cuda", device) if torch.cuda.is_available() else None
        self.exchange = TorchExchange(group, dev)
        self.index.set_shard(self.rank, self.world, self.start, self.n_user_total, (self.exchange.fn, None))

    def rows(self, a):
        """This rank's rows of a per-user array (thresholds, regression records, SVD-space users)."""
        return a[self.start:self.end]

    def query(self, method, query, k_per_q, stats=False):
        """rkr_query over all shards: every rank passes the same queries and gets the whole answer."""
        ks = np.ascontiguousarray(k_per_q, np.int32)
        part, front, st = self.index.shard_query(method, query, ks, stats=True)
        n = front.shape[0]
        gathered = [None] * self.world
        dist.all_gather_object(gathered, (part, front, st), group=self.group)
        parts = [g[0] for g in gathered]
        fronts = [g[1] for g in gathered]
        out, mst = shard_merge(ks[:n], parts, fronts, [g[2] for g in gathered])
        off = np.concatenate([[0], np.cumsum(ks[:n])])
        rows = [out[off[i]:off[i + 1]] for i in range(n)]
        return (rows, mst) if stats else rows


__all__ = ["TorchExchange", "ShardedIndex", "shard_users", "EXCHANGE_FN", "USER_RANK", "QUERY_STATS"]
