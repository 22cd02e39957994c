"""Serving benchmark: a Poisson stream of requests through pk_server.

    python -m pickle_b200.serve_bench [--config c2|c5] [--n N] [--rates 20000,50000,...] [--duration 2]

Each request is one query with k uniform in {10, 50, 100}; arrivals are a
Poisson process at each rate (requests per second).  Two streams per rate:
"mixed", ef uniform in [max(k, 32), 256] (the configuration's range), and
"target", ef = max(k, ef95) where ef95 is the smallest ef of a sweep whose
recall@10 on the query pool (k = 10, one batch) is >= 0.95.  The stream is replayed by the library's native replayer
(pk_server_replay) against a continuous-batching server (slots overlapping on
the GPU, batches of up to --max-batch queries).  Reported per rate: offered
and served requests/s, p50/p99/max latency (submit to results on the host)
and recall@10 of the served results against exact float64 ground truth.
Data are seeded synthetic stand-ins for the configuration's shapes; c5's
768-dimensional rows come from datasets.embedding_like (Zipf-sized clusters,
each spread over its own low-rank subspace, as text embeddings are).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--config", default="c2", choices=["c2", "c5"])
    p.add_argument("--n", type=int, default=0)
    p.add_argument("--pool", type=int, default=20000, help="distinct queries the stream samples from")
    p.add_argument("--rates", default="20000,50000,100000,200000")
    p.add_argument("--duration", type=float, default=2.0, help="seconds of arrivals per rate")
    p.add_argument("--slots", type=int, default=4)
    p.add_argument("--max-batch", type=int, default=4096)
    p.add_argument("--traversal", default="f16", choices=["f16", "fp8"])
    p.add_argument("--M", type=int, default=0)
    p.add_argument("--efc", type=int, default=0)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--streams", default="mixed,target")
    a = p.parse_args(argv)

    import torch

    from pickle_b200 import HNSWIndex, Server, datasets
    from pickle_b200.groundtruth import gpu_knn
    if a.config == "c2":
        n, dim, metric, M, efc = a.n or 1_000_000, 96, "ip", a.M or 32, a.efc or 400
        base, _ = datasets.gmm_unit(n, 0, dim, ncomp=256, sigma=0.3, seed=a.seed)
        _, pool = datasets.gmm_unit(0, a.pool, dim, ncomp=256, sigma=0.3, seed=a.seed)
    else:
        n, dim, metric, M, efc = a.n or 5_000_000, 768, "ip", a.M or 48, a.efc or 200
        base, pool = datasets.embedding_like(n, a.pool, dim, ncomp=2048, zipf_s=1.1, seed=a.seed)
    idx = HNSWIndex(dim, base.dtype, metric, M=M, ef_construction=efc)
    idx.set_seed(a.seed)
    t0 = time.time()
    idx.build(base)
    build_s = time.time() - t0
    idx.prepare_fast(a.traversal)
    gt = gpu_knn(base, pool, 10, metric, torch.device("cuda"))
    # the walk's launch shape, tuned on a full batch of pool queries at the stream's middle ef
    shape, _ = idx.tune_fast(torch.from_numpy(pool[:a.max_batch]).cuda(), 50, 144)
    # recall@10 of the pool at k = 10 over an ef sweep: the stream at the target
    sweep = {}
    ef95 = 1024
    for e in [64, 96, 128, 192, 256, 384, 512, 768, 1024]:
        fi, _ = idx.search_fast(pool, 10, e)
        sweep[e] = round(datasets.recall_at_k(fi, gt, 10), 4)
        if sweep[e] >= 0.95:
            ef95 = e
            break
    print(json.dumps({"config": a.config, "event": "ef_sweep", "k": 10, "recall_at_10": sweep, "ef95": ef95}),
          flush=True)
    srv = Server(idx, a.traversal, slots=a.slots, max_batch=a.max_batch, max_k=100, max_ef=max(512, ef95))
    rng = np.random.default_rng(a.seed + 1)
    for stream in a.streams.split(","):
        for rate in [float(x) for x in a.rates.split(",")]:
            nreq = max(1, int(rate * a.duration))
            arrival = np.cumsum(rng.exponential(1e6 / rate, size=nreq))
            sel = rng.integers(0, len(pool), size=nreq)
            k = rng.choice([10, 50, 100], size=nreq).astype(np.int32)
            if stream == "mixed":
                ef = np.array([rng.integers(max(kk, 32), 257) for kk in k], np.int32)
                ef_desc = "uniform [max(k,32), 256]"
            else:
                ef = np.maximum(k, ef95).astype(np.int32)
                ef_desc = f"max(k, {ef95})"
            ids, _, lat = srv.replay(pool[sel], np.ones(nreq, np.int32), arrival, k, ef, out_stride=100)
            done = arrival / 1e3 + lat
            span_ms = done.max() - arrival[0] / 1e3
            rec = datasets.recall_at_k(ids[:, :10], gt[sel], 10)
            st = srv.stats()
            print(json.dumps({
                "config": a.config, "n": n, "dim": dim, "metric": metric, "M": M, "ef_construction": efc,
                "traversal": a.traversal, "slots": a.slots, "max_batch": a.max_batch, "build_s": round(build_s, 1),
                "launch_shape": shape,
                "offered_req_per_s": rate, "requests": nreq, "served_req_per_s": round(nreq / (span_ms / 1e3), 1),
                "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                               "p99": round(float(np.percentile(lat, 99)), 3), "max": round(float(lat.max()), 3)},
                "stream": stream, "recall_at_10": round(rec, 4), "k": "uniform {10,50,100}", "ef": ef_desc,
                "server": st}), flush=True)
    srv.close()


if __name__ == "__main__":
    main()
