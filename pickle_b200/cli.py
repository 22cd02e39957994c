"""Command-line driver: build an index, search it, sweep k and ef.

Mirrors the reference's benchmark driver (benchmark/hnsw_pickle.cpp and
benchmark/bench_util.hpp): .npy inputs, the same flags where they apply
(--space, --max_degree, --build_ef, --feat_path, --query_path, --label_path,
--index_path, --log_path), the same sweep grid (k in {1, 10, 100}, ef in
{1, 5, ..., 500}, bench_util.hpp:24-25) and the same log line
(hnsw_pickle.cpp:121-122).  Unlike the reference, the index is saved to
--index_path (the reference takes the flag but never writes it) and can be
searched later without rebuilding.

    python -m pickle_b200.cli build  --feat_path X.npy --space l2 --max_degree 32 --build_ef 100 --index_path g.pkg
    python -m pickle_b200.cli search --index_path g.pkg --query_path Q.npy [--label_path L.npy] [--k 10 --ef 48]
    python -m pickle_b200.cli gen    --config c2 --out DIR      # seeded synthetic datasets
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ALL_K = [1, 10, 100]
ALL_EF = [1, 5, 10, 20, 30, 50, 70, 90, 100, 200, 300, 400, 500]


def _log(path, line):
    print(line, flush=True)
    if path:
        with open(path, "a") as f:
            f.write(line + "\n")


def cmd_build(a):
    from pickle_b200 import HNSWIndex
    x = np.load(a.feat_path, mmap_mode="r")
    x = np.ascontiguousarray(x)
    idx = HNSWIndex(x.shape[1], x.dtype, a.space, M=a.max_degree, ef_construction=a.build_ef)
    idx.set_seed(a.seed)
    t0 = time.time()
    idx.build(x, max_batch=a.max_batch)
    dt = time.time() - t0
    idx.save(a.index_path)
    info = idx.info()
    _log(a.log_path, f"BuildTime={dt:.1f}s Nodes={info['n']} Layers={info['num_layers']} "
                     f"DeviceMB={info['device_bytes'] >> 20}")


def cmd_search(a):
    import torch

    from pickle_b200 import HNSWIndex, datasets
    idx = HNSWIndex.load(a.index_path)
    q = np.ascontiguousarray(np.load(a.query_path))
    labels = np.load(a.label_path) if a.label_path else None
    ks = [a.k] if a.k else ALL_K
    efs = [a.ef] if a.ef else ALL_EF
    dev = torch.device("cuda")
    qd = torch.from_numpy(q).to(dev)
    nq = len(q)
    if a.path != "exact":
        idx.prepare_fast(a.path)

    def run(k, ef, ids, ds, counters=None):
        if a.path == "exact":
            idx.search_device(qd, k, ef, ids, ds, counters=counters)
        else:
            idx.search_fast_device(qd, k, ef, ids, ds, counters=counters, expand=a.expand)

    for k in ks:
        for ef in efs:
            if ef < k:
                continue
            ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
            ds = torch.empty((nq, k), dtype=torch.float32, device=dev)
            times = []
            for _ in range(max(1, a.repeat)):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                run(k, ef, ids, ds)
                torch.cuda.synchronize()
                times.append(time.perf_counter() - t0)
            secs = sorted(times)[len(times) // 2]
            cnt = torch.zeros((nq, 6), dtype=torch.int32, device=dev)
            if not a.no_metrics:
                run(k, ef, ids, ds, counters=cnt)
                torch.cuda.synchronize()
            c = cnt.double().sum(0).cpu().numpy() / nq
            recall = 100.0 * datasets.recall_at_k(ids.cpu().numpy(), labels, k) if labels is not None else float("nan")
            # the reference's line: qps/t is per thread; one device counts as one
            _log(a.log_path, f"k={k} search_ef={ef} recall={recall:.1f} qps/t={int(nq / secs)} "
                             f"hop={c[0] + c[3]:.1f} dist={c[1] + c[4]:.1f} base_hop={c[3]:.1f} "
                             f"base_dist={c[4]:.1f} build_ef={idx.ef_construction} thread=1")
            if a.out_ids:
                np.save(a.out_ids, ids.cpu().numpy())


def cmd_gen(a):
    from pickle_b200 import datasets
    os.makedirs(a.out, exist_ok=True)
    if a.config == "c1":
        x, q = datasets.gmm_int_f32(a.n or 100_000, a.nq or 10_000, 128, ncomp=64, sigma=20.0, seed=a.seed)
        metric = "l2"
    elif a.config == "c2":
        x, q = datasets.gmm_unit(a.n or 1_000_000, 0, 96, ncomp=256, sigma=0.3, seed=a.seed)
        _, q = datasets.gmm_unit(0, a.nq or 10_000, 96, ncomp=256, sigma=0.3, seed=a.seed)
        metric = "ip"
    elif a.config in ("c3u8", "c3i8"):
        x, q = datasets.gmm_bytes(a.n or 1_000_000, a.nq or 10_000, 128, ncomp=256, sigma=12.0,
                                  signed=a.config == "c3i8", seed=a.seed)
        metric = "l2"
    elif a.config == "c4":
        x, q = datasets.gmm_f16(a.n or 10_000_000, a.nq or 100_000, 128, ncomp=1024, sigma=0.5, seed=a.seed)
        metric = "l2"
    elif a.config == "c5":
        x, q = datasets.embedding_like(a.n or 5_000_000, a.nq or 10_000, 768, ncomp=2048, zipf_s=1.1, seed=a.seed)
        metric = "ip"
    else:
        raise SystemExit(f"unknown config {a.config}")
    np.save(os.path.join(a.out, "feat.npy"), x)
    np.save(os.path.join(a.out, "query.npy"), q)
    if a.labels:
        from pickle_b200 import datasets as d
        ids, dist = d.exact_knn(x, q, 100, metric)
        np.save(os.path.join(a.out, "label.npy"), ids.astype(np.int32))
        np.save(os.path.join(a.out, "distance.npy"), dist.astype(np.float32))
    print(f"{a.config}: {x.shape} {x.dtype} queries {q.shape} metric={metric} -> {a.out}")


def main(argv=None):
    p = argparse.ArgumentParser(prog="pickle_b200.cli")
    sub = p.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("build")
    b.add_argument("--feat_path", required=True)
    b.add_argument("--space", required=True, choices=["l2", "ip"])
    b.add_argument("--max_degree", type=int, default=32)
    b.add_argument("--build_ef", type=int, default=100)
    b.add_argument("--index_path", required=True)
    b.add_argument("--log_path", default="")
    b.add_argument("--seed", type=int, default=0)
    b.add_argument("--max_batch", type=int, default=0)
    s = sub.add_parser("search")
    s.add_argument("--index_path", required=True)
    s.add_argument("--query_path", required=True)
    s.add_argument("--label_path", default="")
    s.add_argument("--log_path", default="")
    s.add_argument("--k", type=int, default=0)
    s.add_argument("--ef", type=int, default=0)
    s.add_argument("--repeat", type=int, default=3)
    s.add_argument("--no_metrics", action="store_true")
    s.add_argument("--path", default="exact", choices=["exact", "f16", "fp8"],
                   help="exact: the reference's search; f16/fp8: low-precision walk + exact re-rank")
    s.add_argument("--expand", type=int, default=1)
    s.add_argument("--out_ids", default="", help="save the ids of the last (k, ef) searched as .npy")
    g = sub.add_parser("gen")
    g.add_argument("--config", required=True)
    g.add_argument("--out", required=True)
    g.add_argument("--n", type=int, default=0)
    g.add_argument("--nq", type=int, default=0)
    g.add_argument("--seed", type=int, default=0)
    g.add_argument("--labels", action="store_true")
    a = p.parse_args(argv)
    {"build": cmd_build, "search": cmd_search, "gen": cmd_gen}[a.cmd](a)


if __name__ == "__main__":
    sys.exit(main())
