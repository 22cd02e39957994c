"""Multi-GPU layouts (pickle_b200.shard), run as two gloo ranks on the CPU.

The per-rank search is the exact float64 brute force, so each layout's
result can be compared with the single-process answer: integer-valued rows
under L2 make every distance an exact float32 integer, so the merged order
(distance, then id) must equal the single-process order exactly."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from pickle_b200 import datasets, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _brute(base, k):
    def search(q):
        ids, ds = datasets.exact_knn(base, q, k, "l2")
        return ids.astype(np.int32), ds.astype(np.float32)
    return search


def _data(nq):
    return datasets.gmm_int_f32(1500, nq, 16, ncomp=6, sigma=20.0, seed=11)


def _worker(rank, world, port, mode, nq, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        base, queries = _data(nq)
        k = 10
        if mode == "replica":
            ids, ds = shard.replica_search(_brute(base, k), queries, k)
        else:
            lo, hi = shard.query_slice(len(base), rank, world)
            ids, ds = shard.sharded_search(_brute(base[lo:hi], k), queries, k, lo)
        t = shard.max_over_ranks(rank + 0.5)
        np.savez(os.path.join(out_dir, f"{mode}_{rank}.npz"), ids=ids, ds=ds, t=t)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nq", [1, 101])
@pytest.mark.parametrize("mode", ["replica", "sharded"])
def test_two_ranks_match_one_process(mode, nq, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), mode, nq, str(tmp_path)), nprocs=world, join=True)
    base, queries = _data(nq)
    want_i, want_d = datasets.exact_knn(base, queries, 10, "l2")
    for r in range(world):
        got = np.load(tmp_path / f"{mode}_{r}.npz")
        np.testing.assert_array_equal(got["ids"], want_i)
        np.testing.assert_array_equal(got["ds"], want_d.astype(np.float32))
        assert float(got["t"]) == world - 0.5


def test_query_slices_cover_the_batch():
    for nq in [0, 1, 7, 100, 101]:
        for world in [1, 2, 3, 8]:
            parts = [shard.query_slice(nq, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == nq
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.query_slice(10, 2, 2)


def test_merge_topk_orders_by_distance_then_id_and_pads():
    ids = np.array([[[5, 1, -1]], [[2, 9, 1]]], np.int32)          # two shards, one query
    ds = np.array([[[1.0, 3.0, np.inf]], [[1.0, 0.5, 3.0]]], np.float32)
    mi, md = shard.merge_topk(ids, ds, 5)
    np.testing.assert_array_equal(mi, [[9, 2, 5, 1, -1]])          # 1 listed twice is kept once
    np.testing.assert_array_equal(md, [[0.5, 1.0, 1.0, 3.0, np.inf]])


def test_bench_relaunches_itself_for_n_gpus():
    """bench.py --gpus 2 without a torch.distributed environment reruns itself
    under torch.distributed.run with two processes (here on gloo, host only);
    both ranks join and agree on the world size."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                             "MASTER_PORT")}
    p = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--launch-check"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert p.returncode == 0, p.stdout + p.stderr
    line = json.loads([x for x in p.stdout.splitlines() if x.startswith("{")][-1])
    assert line == {"launch_check": True, "world": 2, "ranks_joined": 2}
    # a world size that disagrees with --gpus is refused
    env2 = dict(env, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    q = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--launch-check"],
                       capture_output=True, text=True, timeout=300, env=env2)
    assert q.returncode != 0 and "WORLD_SIZE" in q.stderr
