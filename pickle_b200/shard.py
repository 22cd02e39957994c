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


def merge_topk_tensors(ids, dists, k: int):
    """Merge S candidate lists per query (torch tensors [S, nq, kk], -1 =
    empty) into the k best by (distance, id), ascending, each id once; -1 /
    +inf pad short rows.  Runs where the tensors are (the GPU after an NCCL
    all-gather): two stable sorts give the (distance, id) order, and an id
    listed by two shards (the same row, so the same distance) lands twice in
    a row and keeps its first copy."""
    import torch
    s, nq, kk = ids.shape
    ii = ids.permute(1, 0, 2).reshape(nq, s * kk).to(torch.int64)
    dd = dists.permute(1, 0, 2).reshape(nq, s * kk).to(torch.float64)
    empty = ii < 0
    dd = torch.where(empty, torch.full_like(dd, float("inf")), dd)
    idkey = torch.where(empty, torch.full_like(ii, torch.iinfo(torch.int64).max), ii)
    o1 = torch.argsort(idkey, dim=1, stable=True)
    o2 = torch.argsort(torch.gather(dd, 1, o1), dim=1, stable=True)
    order = torch.gather(o1, 1, o2)
    si = torch.gather(ii, 1, order)
    sd = torch.gather(dd, 1, order)
    drop = si < 0
    drop[:, 1:] |= si[:, 1:] == si[:, :-1]
    keep = torch.argsort(drop.to(torch.int8), dim=1, stable=True)[:, :k]
    out_i = torch.gather(si, 1, keep)
    out_d = torch.gather(sd, 1, keep)
    bad = torch.gather(drop, 1, keep)
    out_i = torch.where(bad, torch.full_like(out_i, -1), out_i).to(torch.int32)
    out_d = torch.where(bad, torch.full_like(out_d, float("inf")), out_d).to(torch.float32)
    if out_i.shape[1] < k:
        pad = k - out_i.shape[1]
        out_i = torch.cat([out_i, torch.full((nq, pad), -1, dtype=torch.int32, device=out_i.device)], 1)
        out_d = torch.cat([out_d, torch.full((nq, pad), float("inf"), device=out_d.device)], 1)
    return out_i, out_d


def merge_topk(ids: np.ndarray, dists: np.ndarray, k: int) -> Tuple[np.ndarray, np.ndarray]:
    """merge_topk_tensors on numpy arrays ([S, nq, kk] each)."""
    import torch
    oi, od = merge_topk_tensors(torch.from_numpy(np.ascontiguousarray(ids)),
                                torch.from_numpy(np.ascontiguousarray(dists)), k)
    return oi.numpy(), od.numpy()


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


def sharded_search_tensors(search, queries, k: int, id_offset: int, group=None):
    """Base-sharded on torch tensors: search(queries) returns this shard's
    (ids int32, dists float32) tensors, [nq, >= k], ids local to the shard;
    they are shifted by id_offset to global ids, every shard's top-k is
    all-gathered (one NCCL all_gather per array on GPU tensors, over
    NVLink/NVSwitch; gloo on CPU tensors) and merged where the tensors are.
    Every rank returns the merged (ids, dists)."""
    import torch
    import torch.distributed as dist
    ids, ds = search(queries)
    ids = ids[:, :k].to(torch.int64)
    ids = torch.where(ids >= 0, ids + id_offset, torch.full_like(ids, -1)).to(torch.int32).contiguous()
    ds = ds[:, :k].to(torch.float32).contiguous()
    world = dist.get_world_size(group)
    all_i = [torch.empty_like(ids) for _ in range(world)]
    all_d = [torch.empty_like(ds) for _ in range(world)]
    dist.all_gather(all_i, ids, group=group)
    dist.all_gather(all_d, ds, group=group)
    return merge_topk_tensors(torch.stack(all_i), torch.stack(all_d), k)


def sharded_search(search: SearchFn, queries: np.ndarray, k: int, id_offset: int, group=None):
    """Base-sharded with numpy in and out: search the whole batch on this
    rank's shard, all-gather and merge as sharded_search_tensors does (on the
    rank's GPU for NCCL groups).  Every rank returns the merged result."""
    import torch
    dev = _comm_device(group)

    def run(q):
        i, d = search(q.cpu().numpy())
        return torch.from_numpy(np.ascontiguousarray(i)).to(dev), torch.from_numpy(np.ascontiguousarray(d)).to(dev)

    oi, od = sharded_search_tensors(run, torch.from_numpy(np.ascontiguousarray(queries)), k, id_offset, group)
    return oi.cpu().numpy(), od.cpu().numpy()


def max_over_ranks(value: float, group=None) -> float:
    """The largest of every rank's value (device timings are reported as the
    maximum over ranks)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=_comm_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
