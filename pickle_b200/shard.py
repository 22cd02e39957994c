"""Multi-GPU search over torch.distributed: one process per GPU, two layouts.

Replicas (query-sharded): every rank holds the whole index and answers a
contiguous slice of the batch.  The search itself needs no collective; the
slices are gathered only when every rank wants the whole result.

Base-sharded: rank r holds the rows [offset_r, offset_r + n_r) as its own
index; every rank searches the whole batch on its shard, the per-shard top-k
(ids mapped to global ids, distances) are all-gathered, and each query's
lists are merged by (distance, id).  Recall then differs from one graph over
all rows, and is reported separately.

The reference is single-process (OpenMP inside one AnnSearch call,
include/hnsw.hpp:528-541); this is the layer above it.  Collectives run on
NCCL for GPU process groups (tensors on the rank's device; NVLink/NVSwitch)
and on gloo for CPU groups.  A search function maps a query block to
(ids int32 [n, k], dists float32 [n, k]) with -1 / +inf padding, for example
HNSWIndex.search or search_fast.
"""
from __future__ import annotations

from typing import Callable, Tuple

import numpy as np

SearchFn = Callable[[np.ndarray], Tuple[np.ndarray, np.ndarray]]


def query_slice(nq: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous balanced slice [lo, hi) of nq queries for rank of world
    (the first nq % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(nq, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def merge_topk(ids: np.ndarray, dists: np.ndarray, k: int) -> Tuple[np.ndarray, np.ndarray]:
    """Merge S candidate lists per query ([S, nq, kk] each, -1 = empty) into
    the k best by (distance, id), ascending; -1 / +inf pad short rows."""
    s, nq, kk = ids.shape
    ii = np.transpose(ids, (1, 0, 2)).reshape(nq, s * kk).astype(np.int64)
    dd = np.transpose(dists, (1, 0, 2)).reshape(nq, s * kk).astype(np.float64)
    dd = np.where(ii < 0, np.inf, dd)
    ii_key = np.where(ii < 0, np.iinfo(np.int64).max, ii)
    out_i = np.full((nq, k), -1, np.int32)
    out_d = np.full((nq, k), np.inf, np.float32)
    for r in range(nq):
        order = np.lexsort((ii_key[r], dd[r]))
        seen = set()
        j = 0
        for c in order:
            if ii[r, c] < 0 or j == k:
                break
            if ii[r, c] in seen:
                continue
            seen.add(int(ii[r, c]))
            out_i[r, j] = ii[r, c]
            out_d[r, j] = dd[r, c]
            j += 1
    return out_i, out_d


def _comm_device(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _all_gather_rows(x: np.ndarray, group=None) -> list:
    """All-gather row blocks of possibly different lengths (same trailing
    shape and type) from every rank; returns the list of blocks by rank."""
    import torch
    import torch.distributed as dist
    dev = _comm_device(group)
    world = dist.get_world_size(group)
    n = torch.tensor([x.shape[0]], dtype=torch.int64, device=dev)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    ns = [int(v.item()) for v in ns]
    m = max(ns) if ns else 0
    pad = np.zeros((m,) + x.shape[1:], x.dtype)
    pad[: x.shape[0]] = x
    t = torch.from_numpy(pad).to(dev)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    return [o.cpu().numpy()[:c] for o, c in zip(outs, ns)]


def replica_search(search: SearchFn, queries: np.ndarray, k: int, group=None, gather: bool = True):
    """Replicas: this rank answers its slice of the batch.  With gather, every
    rank returns the whole batch's (ids, dists); otherwise this rank's slice
    and its [lo, hi)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = query_slice(len(queries), rank, world)
    ids, ds = search(queries[lo:hi]) if hi > lo else (np.empty((0, k), np.int32), np.empty((0, k), np.float32))
    ids, ds = np.ascontiguousarray(ids[:, :k], np.int32), np.ascontiguousarray(ds[:, :k], np.float32)
    if not gather:
        return ids, ds, (lo, hi)
    return np.concatenate(_all_gather_rows(ids, group)), np.concatenate(_all_gather_rows(ds, group))


def sharded_search(search: SearchFn, queries: np.ndarray, k: int, id_offset: int, group=None):
    """Base-sharded: search the whole batch on this rank's shard (ids local to
    the shard, shifted by id_offset to global ids), all-gather every shard's
    top-k, merge by (distance, id).  Every rank returns the merged result."""
    ids, ds = search(queries)
    ids = np.where(ids[:, :k] >= 0, ids[:, :k].astype(np.int64) + id_offset, -1).astype(np.int32)
    ds = np.ascontiguousarray(ds[:, :k], np.float32)
    all_i = np.stack(_all_gather_rows(np.ascontiguousarray(ids), group))
    all_d = np.stack(_all_gather_rows(ds, group))
    return merge_topk(all_i, all_d, k)


def max_over_ranks(value: float, group=None) -> float:
    """The largest of every rank's value (device timings are reported as the
    maximum over ranks)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_comm_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
