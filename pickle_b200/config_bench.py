"""Search benchmark over the configurations beyond the headline one.

    python -m pickle_b200.config_bench --config c1|c3u8|c3i8|c4 [--paths exact,f16,fp8] [--n N] [--nq NQ]
                                       [--cpu-sample Q]

Each configuration is a seeded synthetic stand-in with the shape, type,
metric and graph parameters of one of the reference's benchmark datasets
(the public files are not available offline):

  c1    100k x 128 integer-valued float32 (64-component mixture, centres in
        [0, 255], sigma 20, rounded and clipped), L2, M=16, efC=200,
        10k queries, k=10, ef in {16, 32, 64, 128, 256}
  c3u8  1M x 128 uint8 (sigma 12), L2 in int32, M=16, efC=200, 10k queries
  c3i8  the same in int8
  c4    10M x 128 float16 (1024-component mixture, sigma 0.5), L2, M=32,
        efC=200, 100k queries each with its own k in {1, 10, 100} and ef
        uniform in [max(k, 16), 512] (one mixed batch), then the same
        queries at k=10 over an ef sweep (the recall@10 >= 0.95 point)

The index is built on the GPU.  Per path (exact = the reference's search;
f16 / fp8 = low-precision walk plus exact re-rank, launch shape tuned on the
batch) and ef, one JSON line: queries/s from CUDA events around whole
batches (L2 flushed before each batch, median of the timed batches),
recall@k against exact float64 ground truth, per-query distance evaluations, the relative error of the returned
distances against float64 (the re-rank is exact in FP32 or integers), and
for the fast paths the relative error of the traversal copy's distances to
each query's true neighbours (restated on the host by the library's scaling
rules).
With --cpu-sample, the reference's own search (the oracle harness built from
the reference sources, when present) is timed on the saved graph on all host
threads for a sample of the queries at one ef.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

CONFIGS = {
    "c1": dict(n=100_000, nq=10_000, dim=128, metric="l2", M=16, efc=200, efs=[16, 32, 64, 128, 256]),
    "c3u8": dict(n=1_000_000, nq=10_000, dim=128, metric="l2", M=16, efc=200, efs=[16, 32, 64, 128, 256]),
    "c3i8": dict(n=1_000_000, nq=10_000, dim=128, metric="l2", M=16, efc=200, efs=[16, 32, 64, 128, 256]),
    "c4": dict(n=10_000_000, nq=100_000, dim=128, metric="l2", M=32, efc=200, efs=[16, 24, 32, 48, 64, 96, 112, 128],
               mixed=True),
}


def make(cfg_name, n, nq, seed):
    from pickle_b200 import datasets
    c = CONFIGS[cfg_name]
    if cfg_name == "c1":
        return datasets.gmm_int_f32(n, nq, c["dim"], ncomp=64, sigma=20.0, seed=seed)
    if cfg_name in ("c3u8", "c3i8"):
        return datasets.gmm_bytes(n, nq, c["dim"], ncomp=256, sigma=12.0, signed=cfg_name == "c3i8", seed=seed)
    return datasets.gmm_f16(n, nq, c["dim"], ncomp=1024, sigma=0.5, seed=seed)


def exact_dist(base, queries, ids, metric):
    """float64 distances (index convention) of queries[i] to base[ids[i, j]]."""
    q = queries.astype(np.float64)[:, None, :]
    rows = base[np.maximum(ids, 0)].astype(np.float64)
    return -(q * rows).sum(-1) if metric == "ip" else ((q - rows) ** 2).sum(-1)


def traversal_copy(base, queries, path):
    """The traversal copy the library walks with, restated on the host by the
    same rules: FP16 = values divided by the power of two sc with
    max|x| / sc in [4, 8) (queries clamped to 64 in those units); FP8 E4M3 =
    values divided by per-dimension max|x| / 448, rounded to E4M3 and scaled
    back (queries in full precision: the kernel's two E4M3 query parts carry a
    component to 0.04%, median, and 0.2% at worst).  Returns (rows, queries) as float64
    in original units."""
    import torch
    amax = np.abs(base.astype(np.float32)).max(0)
    if path == "f16":
        mx = float(amax.max())
        sc = 2.0 ** np.frexp(mx / 8.0)[1] if mx > 0 else 1.0
        r = (base.astype(np.float32) / sc).astype(np.float16).astype(np.float64) * sc
        qq = np.clip(queries.astype(np.float32) / sc, -64, 64).astype(np.float16).astype(np.float64) * sc
        return r, qq
    scale = np.where(amax > 0, amax / 448.0, 1.0).astype(np.float32)
    e = torch.from_numpy(base.astype(np.float32) / scale).to(torch.float8_e4m3fn).float().numpy()
    return e.astype(np.float64) * scale, queries.astype(np.float64)


def traversal_error(base, queries, gt, metric, path, nsample=1000):
    """Relative error of traversal distances (median, 99th percentile) over
    each sampled query's 10 true nearest rows; L2 is evaluated as the kernels
    do, |q|^2 + |x|^2 - 2 q.x from the stored values."""
    ids = gt[:nsample, :10]
    sel = np.unique(ids)
    rows_t, q_t = traversal_copy(base[sel], queries[:nsample], path)
    pos = np.searchsorted(sel, ids)
    rt = rows_t[pos]
    qt = q_t[:, None, :]
    if metric == "ip":
        dt = -(qt * rt).sum(-1)
    else:
        dt = (qt * qt).sum(-1) + (rt * rt).sum(-1) - 2.0 * (qt * rt).sum(-1)
    de = exact_dist(base, queries[:nsample], ids, metric)
    rel = np.abs(dt - de) / np.maximum(np.abs(de), 1e-30)
    return float(np.median(rel)), float(np.percentile(rel, 99))


def recall_mixed(found, truth, ks):
    hit = 0
    for f, t, k in zip(found, truth, ks):
        hit += len(set(int(x) for x in f[:k] if x >= 0) & set(int(x) for x in t[:k]))
    return hit / float(np.sum(ks))


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--config", required=True, choices=sorted(CONFIGS))
    p.add_argument("--paths", default="exact,f16,fp8")
    p.add_argument("--n", type=int, default=0)
    p.add_argument("--nq", type=int, default=0)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--cpu-sample", type=int, default=0, help="queries timed on the reference's CPU search")
    p.add_argument("--efs", default="", help="comma-separated ef list instead of the configuration's sweep")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed k/ef batch")
    p.add_argument("--fast-shape", default="", help="rows,filter_log2,warps for the fast walk instead of tuning")
    a = p.parse_args(argv)

    import torch

    from pickle_b200 import HNSWIndex, datasets
    from pickle_b200.groundtruth import gpu_knn
    c = CONFIGS[a.config]
    n, nq = a.n or c["n"], a.nq or c["nq"]
    t0 = time.time()
    base, queries = make(a.config, n, nq, a.seed)
    gen_s = time.time() - t0
    idx = HNSWIndex(c["dim"], base.dtype, c["metric"], M=c["M"], ef_construction=c["efc"])
    idx.set_seed(a.seed)
    torch.cuda.synchronize()
    t0 = time.time()
    idx.build(base)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    info = idx.info()
    dev = torch.device("cuda")
    mixed = c.get("mixed", False) and not a.no_mixed
    ef_list = [int(x) for x in a.efs.split(",")] if a.efs else c["efs"]
    kmax = 100 if mixed else 10
    t0 = time.time()
    gt = gpu_knn(base, queries, kmax, c["metric"], dev)
    gt_s = time.time() - t0
    head = {"config": a.config, "n": n, "nq": nq, "dim": c["dim"], "dtype": str(base.dtype), "metric": c["metric"],
            "M": c["M"], "ef_construction": c["efc"], "gen_s": round(gen_s, 1), "build_s": round(build_s, 1),
            "gt_s": round(gt_s, 1), "device_mb": info["device_bytes"] >> 20}
    print(json.dumps(dict(head, event="built")), flush=True)

    q = torch.from_numpy(queries).to(dev)
    rng = np.random.default_rng(a.seed + 7)
    k10 = np.full(nq, 10, np.int32)
    # (label, k, ef, per-query k on the host, per-query k / ef on the device)
    runs = []
    if mixed:
        kq = rng.choice([1, 10, 100], size=nq).astype(np.int32)
        efq = np.array([rng.integers(max(int(k), 16), 513) for k in kq], np.int32)
        runs.append(("mixed", int(kq.max()), int(efq.max()), kq, torch.from_numpy(kq).to(dev),
                     torch.from_numpy(efq).to(dev)))
    runs += [(str(e), 10, e, k10, None, None) for e in ef_list]
    stride = max(r[1] for r in runs)
    ids = torch.empty((nq, stride), dtype=torch.int32, device=dev)
    ds = torch.empty((nq, stride), dtype=torch.float32, device=dev)
    cnt = torch.zeros((nq, 6), dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def call(path, k, ef, k_dev, ef_dev, counters=None):
        if path == "exact":
            idx.search_device(q, k, ef, ids, ds, k_per_query=k_dev, ef_per_query=ef_dev, counters=counters)
        else:
            idx.search_fast_device(q, k, ef, ids, ds, k_per_query=k_dev, ef_per_query=ef_dev, counters=counters)

    for path in a.paths.split(","):
        if path != "exact":
            idx.prepare_fast(path)
        for label, k, ef, ks, k_dev, ef_dev in runs:
            if path != "exact" and ef > 512:
                continue
            shape = None
            if path != "exact":
                if a.fast_shape:
                    shape = tuple(int(x) for x in a.fast_shape.split(","))
                    idx.set_fast_params(*shape)
                else:
                    shape, _ = idx.tune_fast(q, k, min(ef, 512))
            call(path, k, ef, k_dev, ef_dev)
            torch.cuda.synchronize()
            times = []
            for step in range(a.steps + 1):
                flush.fill_(1)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                call(path, k, ef, k_dev, ef_dev)
                e1.record()
                e1.synchronize()
                if step:
                    times.append(e0.elapsed_time(e1))
            ms = float(np.median(times))
            got = ids.cpu().numpy()
            rec = recall_mixed(got, gt, ks)
            # returned distances against float64 for the returned ids (a sample)
            ns = min(nq, 2000)
            gd = ds.cpu().numpy()[:ns, :10]
            # a row holds results up to its own k only
            ok = (got[:ns, :10] >= 0) & (np.arange(10)[None, :] < ks[:ns, None])
            gi = np.where(ok, got[:ns, :10], 0)
            ex = exact_dist(base, queries[:ns], gi, c["metric"])
            rel = np.abs(gd - ex)[ok] / np.maximum(np.abs(ex[ok]), 1e-30)
            dist_err = {"max_rel": float(rel.max()), "median_rel": float(np.median(rel))}
            trav_err = None
            if path != "exact":
                med, p99 = traversal_error(base, queries, gt, c["metric"], path)
                trav_err = {"median_rel": med, "p99_rel": p99}
            cnt.zero_()
            call(path, k, ef, k_dev, ef_dev, counters=cnt)
            torch.cuda.synchronize()
            cc = cnt.double().mean(0).cpu().numpy()
            print(json.dumps(dict(head, event="search", path=path, ef=label,
                                  k=("mixed {1,10,100}" if label == "mixed" else k),
                                  qps=round(nq / ms * 1e3, 1), ms_per_batch=round(ms, 3), recall=round(rec, 4),
                                  dist_per_query=round(float(cc[1] + cc[4]), 1),
                                  hops_l0=round(float(cc[3]), 1), launch_shape=shape, returned_dist_err=dist_err,
                                  traversal_dist_err=trav_err)), flush=True)

    if a.cpu_sample:
        import oracle
        if oracle.ref_available():
            ef = 64
            with tempfile.TemporaryDirectory() as td:
                gp = os.path.join(td, "g.pkg")
                idx.save(gp)
                sample = queries[:a.cpu_sample]
                threads = os.cpu_count() or 1
                _, _, ci = oracle.ref_search(gp, sample, 10, ef, threads=threads, repeat=3, want_results=False)
            print(json.dumps(dict(head, event="cpu_reference", ef=ef, k=10, qps=round(ci["qps"], 1), cores=threads,
                                  sample=len(sample))), flush=True)


if __name__ == "__main__":
    main()
