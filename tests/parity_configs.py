"""Search parity at the benchmark configurations' full size (GPU + host).

    python -m tests.parity_configs --config c2|c3u8|c3i8|c5sub [--build] [--nq N] [--efs 32,64] [--ks 10,100]

Test infrastructure, run by hand on a GPU machine (its output is summarised
under profiles/): too long for the unit-test suite.  For each configuration
the graph is built by the reference's own parallel Build on all host cores
(oracle/_ref/pk_ref), then at every (k, ef) the device's exact search
(pk_index_search_device) and the reference binary's batch AnnSearch answer the
same queries on that file:

  c3u8 / c3i8  1M x 128 uint8 / int8 (256-component mixture, sigma 12), L2 in
               int32, M = 16, efC = 200: ids, distances and the per-level work
               counters must be equal bit for bit.
  c2           1M x 96 float32 unit rows (256-component mixture, sigma 0.3),
               inner product, M = 32, efC = 400: the restatement replayed with
               the device's float summation order must return exactly the
               device's ids and distances; the queries whose ids differ from
               the reference binary's beyond ties within 1e-6 relative are
               counted, and each is replayed by the fork detector (the
               device's distances driving, the reference binary's own
               distances compared at every decision) to find the comparison
               where the two searches part; recall@k against exact float64
               ground truth must agree within 0.001.

With --build the configuration's graph is built --seeds times by the device
(pk_index_build, batched insertion on the GPU, seeds 0 ..) and as many times
by the reference's parallel Build (level draws from seeds 0 ..), and every
graph is searched by the reference binary's AnnSearch at every ef.  Two
graphs of the same data differ in recall by more than the sampling error of
one recall (which graph a seed draws matters), so the check compares the
mean recall of the device graphs with the reference graphs' mean, within two
standard errors of the difference: the spread of each side's graphs over
its seeds plus the sampling error of a recall over nq x 10 labels.

One JSON line per (k, ef); exit status 1 if any check fails.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CONFIGS = {
    "c2": dict(n=1_000_000, nq=10_000, dim=96, metric="ip", M=32, efc=400, efs=[32, 64, 128, 256, 512], ks=[10, 100]),
    "c3u8": dict(n=1_000_000, nq=10_000, dim=128, metric="l2", M=16, efc=200, efs=[16, 32, 64, 128, 256], ks=[10]),
    "c3i8": dict(n=1_000_000, nq=10_000, dim=128, metric="l2", M=16, efc=200, efs=[16, 32, 64, 128, 256], ks=[10]),
    # a 500k-row subset of the serving configuration (768-dimensional float16
    # embedding-like rows, inner product, M = 48), for --build
    "c5sub": dict(n=500_000, nq=2_000, dim=768, metric="ip", M=48, efc=200, efs=[64, 128, 256, 512], ks=[10]),
}


def make(name, n, nq, seed):
    from pickle_b200 import datasets
    if name == "c2":
        return datasets.gmm_unit(n, nq, 96, ncomp=256, sigma=0.3, seed=seed)
    if name == "c5sub":
        return datasets.embedding_like(n, nq, 768, ncomp=2048, zipf_s=1.1, seed=seed)
    return datasets.gmm_bytes(n, nq, 128, ncomp=256, sigma=12.0, signed=name == "c3i8", seed=seed)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--config", required=True, choices=sorted(CONFIGS))
    p.add_argument("--n", type=int, default=0)
    p.add_argument("--nq", type=int, default=0)
    p.add_argument("--efs", default="")
    p.add_argument("--ks", default="")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--build", action="store_true", help="compare the device build with the reference build")
    p.add_argument("--seeds", type=int, default=1, help="graphs built per side with --build")
    p.add_argument("--max-fork-queries", type=int, default=100,
                   help="mismatched float queries replayed by the fork detector per (k, ef)")
    a = p.parse_args(argv)

    import torch

    import oracle
    from pickle_b200 import HNSWIndex, datasets
    from pickle_b200.groundtruth import gpu_knn
    from tests.helpers import mismatched_queries, reference_distance_table

    c = CONFIGS[a.config]
    n, nq = a.n or c["n"], a.nq or c["nq"]
    efs = [int(x) for x in a.efs.split(",")] if a.efs else c["efs"]
    ks = [int(x) for x in a.ks.split(",")] if a.ks else c["ks"]
    base, queries = make(a.config, n, nq, a.seed)
    integer = base.dtype in (np.uint8, np.int8)
    ok_all = True
    with tempfile.TemporaryDirectory() as td:
        head = {"config": a.config, "n": n, "nq": nq, "dim": c["dim"], "dtype": str(base.dtype),
                "metric": c["metric"], "M": c["M"], "ef_construction": c["efc"]}
        if a.build:
            from tests.helpers import build_recall_tolerance, levels_for
            gt_b = gpu_knn(base, queries, 10, c["metric"], torch.device("cuda"))
            rec = {"reference": {ef: [] for ef in efs}, "device": {ef: [] for ef in efs}}
            for seed in range(a.seeds):
                rpath, dpath = os.path.join(td, "ref.pkg"), os.path.join(td, "dev.pkg")
                t0 = time.time()
                oracle.ref_build(base, c["metric"], c["M"], c["efc"], rpath,
                                 levels=levels_for(n, c["M"], seed) if a.seeds > 1 else None)
                ref_s = time.time() - t0
                t0 = time.time()
                dev_idx = HNSWIndex(c["dim"], base.dtype, c["metric"], M=c["M"], ef_construction=c["efc"])
                dev_idx.set_seed(a.seed + seed)
                dev_idx.build(base)
                torch.cuda.synchronize()
                dev_s = time.time() - t0
                dev_idx.save(dpath)
                dev_idx.close()
                line = dict(head, event="built", seed=seed, ref_build_s=round(ref_s, 1), device_build_s=round(dev_s, 1))
                for ef in efs:
                    rr, _, _ = oracle.ref_search(rpath, queries, 10, ef)
                    rd, _, _ = oracle.ref_search(dpath, queries, 10, ef)
                    rec["reference"][ef].append(datasets.recall_at_k(rr, gt_b, 10))
                    rec["device"][ef].append(datasets.recall_at_k(rd, gt_b, 10))
                    line[f"recall_ef{ef}"] = [round(rec["reference"][ef][-1], 5), round(rec["device"][ef][-1], 5)]
                print(json.dumps(line), flush=True)
            for ef in efs:
                r_ref, r_dev = np.array(rec["reference"][ef]), np.array(rec["device"][ef])
                m_ref, m_dev = float(r_ref.mean()), float(r_dev.mean())
                tol = build_recall_tolerance(r_ref, r_dev, 10 * nq)
                ok = m_dev >= m_ref - tol
                ok_all &= bool(ok)
                print(json.dumps(dict(head, event="build_recall", ef=ef, k=10, graphs_per_side=a.seeds,
                                      recall_reference_graphs=[round(x, 5) for x in r_ref],
                                      recall_device_graphs=[round(x, 5) for x in r_dev],
                                      mean_reference=round(m_ref, 5), mean_device=round(m_dev, 5),
                                      tolerance=round(tol, 5), ok=bool(ok))), flush=True)
            return 0 if ok_all else 1
        path = os.path.join(td, "ref.pkg")
        t0 = time.time()
        binfo = oracle.ref_build(base, c["metric"], c["M"], c["efc"], path)
        build_s = time.time() - t0
        head.update(ref_build_s=round(build_s, 1), ref_build_threads=binfo.get("threads"))
        print(json.dumps(dict(head, event="built")), flush=True)
        idx = HNSWIndex.load(path)
        g = oracle.OraGraph.load(path)
        dev = torch.device("cuda")
        q = torch.from_numpy(queries).to(dev)
        gt = gpu_knn(base, queries, max(ks), c["metric"], dev)
        for k in ks:
            for ef in efs:
                if ef < k:
                    continue
                ri, rd, info = oracle.ref_search(path, queries, k, ef, metrics=True)
                ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
                ds = torch.empty((nq, k), dtype=torch.float32, device=dev)
                cnt = torch.zeros((nq, 6), dtype=torch.int32, device=dev)
                idx.search_device(q, k, ef, ids, ds, counters=cnt)
                torch.cuda.synchronize()
                ids, ds = ids.cpu().numpy(), ds.cpu().numpy()
                cnt = cnt.cpu().numpy().astype(np.int64)
                counters_equal = bool(cnt[:, 0].sum() + cnt[:, 3].sum() == info["hop"] and
                                      cnt[:, 1].sum() + cnt[:, 4].sum() == info["dist"] and
                                      cnt[:, 3].sum() == info["base_hop"] and cnt[:, 4].sum() == info["base_dist"] and
                                      cnt[:, 2].sum() + cnt[:, 5].sum() == info["neighbor"])
                r_dev = datasets.recall_at_k(ids, gt, k)
                r_ref = datasets.recall_at_k(ri, gt, k)
                line = dict(head, event="parity", k=k, ef=ef, recall_device=round(r_dev, 5),
                            recall_reference=round(r_ref, 5))
                if integer:
                    ids_equal = bool(np.array_equal(ids, ri))
                    dists_equal = bool(np.array_equal(ds, rd))
                    ok = ids_equal and dists_equal and counters_equal
                    line.update(ids_equal=ids_equal, dists_equal=dists_equal, counters_equal=counters_equal,
                                queries_differing=int((ids != ri).any(1).sum()))
                else:
                    with oracle.float_order(oracle.ORDER_DEVICE):
                        oi, od = g.search(queries, k, ef)
                    replay_equal = bool(np.array_equal(ids, oi) and np.array_equal(ds, od))
                    bad = mismatched_queries(ids, ds, ri, rd)
                    forks, gaps = [], []
                    sel = bad[: a.max_fork_queries]
                    if sel:
                        qs = np.ascontiguousarray(queries[sel])
                        _, _, _, touched = g.search_fork(qs, k, ef, oracle.ORDER_DEVICE, oracle.ORDER_DEVICE,
                                                         touched_cap=400_000)
                        table = reference_distance_table(base, qs, touched, c["metric"])
                        _, _, fork, _ = g.search_fork(qs, k, ef, oracle.ORDER_DEVICE, oracle.ORDER_TABLE, table=table)
                        for f in fork:
                            forks.append(int(f[1]) if f[0] else 0)
                            if f[0]:
                                ga = abs(f[2] - f[3]) / max(abs(f[2]), abs(f[3]), 1e-30)
                                gb = abs(f[4] - f[5]) / max(abs(f[4]), abs(f[5]), 1e-30)
                                gaps.append(min(ga, gb))
                    all_forked = all(w in (1, 2, 3, 4) for w in forks)
                    max_gap = max(gaps) if gaps else 0.0
                    recall_ok = abs(r_dev - r_ref) <= 0.001 + 1.0 / (k * nq)
                    ok = replay_equal and all_forked and recall_ok and max_gap <= 1e-6
                    line.update(device_order_replay_equal=replay_equal, queries_differing=int((ids != ri).any(1).sum()),
                                mismatched_beyond_ties=len(bad), fork_replayed=len(sel),
                                fork_where={w: forks.count(w) for w in sorted(set(forks))},
                                max_fork_gap=max_gap, median_fork_gap=float(np.median(gaps)) if gaps else 0.0,
                                counters_equal=counters_equal)
                line["ok"] = bool(ok)
                ok_all &= bool(ok)
                print(json.dumps(line), flush=True)
    return 0 if ok_all else 1


if __name__ == "__main__":
    sys.exit(main())
