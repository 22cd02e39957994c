"""QPS at recall@10 >= 0.95 for HNSW search on one B200 (and N replicas).

Workload (the configuration the headline metric is quoted on): 1M base
vectors, dim 96, float32, unit-normalised rows from a 256-component Gaussian
mixture (sigma 0.3 around random unit centres), inner product, M = 32,
ef_construction = 400; 10k queries from the same mixture, k = 10.  Data are
seeded synthetic stand-ins (the public datasets are not available offline).
ef is the smallest value of a fixed sweep whose recall@10 against exact
(float64) ground truth reaches 0.95.

A step is one batch search of the 10k queries.
  value   device-resident: queries and results in HBM, CUDA events around each
          pk_index_search_device call on its stream, L2 flushed between steps.
  e2e     through the C ABI with host buffers (pk_index_search): pinned host
          queries in, ids and distances out, copies inside the timed region.
  roofline  algorithmic bytes per launch (distance rows read + adjacency rows
          read, from the device's own work counters) over the kernel's average
          duration, against the measured HBM copy bandwidth.
  cpu_baseline  the reference's own search (oracle/_ref/pk_ref, all host
          threads) on the same saved graph, on a bounded sample of the queries.

--impl reference runs the reference's own build and search on the host cores
instead (rank 0 only) and prints the same line with impl = reference.

Multi-GPU (torchrun, one process per GPU): every rank holds a full replica and
searches its own 10k queries; no collective is on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC_NAME = "QPS at recall@10>=0.95 (1M x 96 f32, IP, M=32, efC=400, k=10)"
EF_SWEEP = [16, 24, 32, 36, 40, 44, 48, 56, 64, 80, 96, 112, 128, 160, 192, 256, 320, 384, 512]
RECALL_TARGET = 0.95


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=1_000_000)
    p.add_argument("--nq", type=int, default=10_000)
    p.add_argument("--dim", type=int, default=96)
    p.add_argument("--M", type=int, default=32)
    p.add_argument("--efc", type=int, default=400)
    p.add_argument("--k", type=int, default=10)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-sample", type=int, default=2000, help="queries in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--paths", default="exact,f16,fp8", help="search paths to measure (exact, f16, fp8)")
    p.add_argument("--expand", type=int, default=1, help="entries expanded per step on the fast paths")
    p.add_argument("--fast-shape", default="", help="rows,filter_log2,warps for the fast walk instead of tuning")
    return p.parse_args()


def log(args, *a):
    if args.verbose:
        print(*a, file=sys.stderr, flush=True)


def make_data(args, rank):
    from pickle_b200 import datasets
    base, _ = datasets.gmm_unit(args.n, 0, args.dim, ncomp=256, sigma=0.3, seed=args.seed)
    # every rank has its own 10k queries from the same mixture
    _, queries = datasets.gmm_unit(0, args.nq, args.dim, ncomp=256, sigma=0.3, seed=args.seed)
    if rank:
        rng = np.random.default_rng(1000 + rank)
        queries = queries[rng.permutation(len(queries))]
    return base, queries


def ground_truth(base, queries, k, device):
    """Exact top-k by inner product: float32 candidates, float64 rescoring."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    b = torch.from_numpy(base).to(device)
    out = np.empty((len(queries), k), np.int64)
    cand = 64
    for i in range(0, len(queries), 1024):
        q = torch.from_numpy(queries[i:i + 1024]).to(device)
        s = q @ b.T
        top = torch.topk(s, cand, dim=1).indices
        s64 = (q.double()[:, None, :] * b[top].double()).sum(-1)
        order = torch.argsort(-s64, dim=1, stable=True)[:, :k]
        out[i:i + 1024] = torch.gather(top, 1, order).cpu().numpy()
    del b
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic_per_query(kernel):
    """DRAM bytes per query of a kernel from its committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", f"{kernel}_1Mx96_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def cpu_baseline(args, graph_path, queries, ef):
    """The reference's AnnSearch on the saved graph, all host threads, on a bounded sample."""
    import oracle
    if not oracle.ref_available():
        return None
    sample = queries[: args.cpu_sample]
    threads = os.cpu_count() or 1
    _, _, info = oracle.ref_search(graph_path, sample, args.k, ef, threads=threads, repeat=3, want_results=False)
    return {"value": round(info["qps"], 1), "unit": "queries/s", "cores": threads, "kind": "reference",
            "sample": f"{len(sample)} of the {len(queries)} queries at ef={ef}, same graph file, median of 3 batch "
                      f"AnnSearch runs (steady clock around the batch)"}


def run_ours(args):
    import ctypes

    import torch
    import torch.distributed as dist

    from pickle_b200 import HNSWIndex, datasets, lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=30), device_id=dev)

    base, queries = make_data(args, rank)
    log(args, f"[{rank}] data ready")
    idx = HNSWIndex(args.dim, np.float32, "ip", M=args.M, ef_construction=args.efc)
    idx.set_seed(args.seed)
    t0 = time.time()
    idx.build(base)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    log(args, f"[{rank}] build {build_s:.1f}s")
    gt = ground_truth(base, queries, args.k, dev)

    nq, k = len(queries), args.k
    q_dev = torch.from_numpy(queries).to(dev)
    ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    ds = torch.empty((nq, k), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MiB > 126 MB of L2
    L = lib()
    qh = torch.from_numpy(queries).pin_memory()
    ih = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    dh = torch.empty((nq, k), dtype=torch.float32).pin_memory()

    def call(path, ef, counters=None):
        if path == "exact":
            idx.search_device(q_dev, k, ef, ids, ds, counters=counters, stream=stream)
        else:
            idx.search_fast_device(q_dev, k, ef, ids, ds, counters=counters, expand=args.expand, stream=stream)

    def host_call(path, ef):
        qp, ip_, dp = (ctypes.c_void_p(t.data_ptr()) for t in (qh, ih, dh))
        if path == "exact":
            rc = L.pk_index_search(idx._h, qp, nq, k, ef, ip_, dp)
        else:
            rc = L.pk_index_search_fast_host(idx._h, qp, nq, k, ef, ip_, dp, args.expand)
        if rc != 0:
            raise RuntimeError(L.pk_last_error().decode())

    def measure(path):
        if path != "exact":
            idx.prepare_fast(path)
        ef, recall, sweep = None, 0.0, {}
        for e in EF_SWEEP:
            call(path, e)
            torch.cuda.synchronize()
            r = datasets.recall_at_k(ids.cpu().numpy(), gt, k)
            sweep[e] = round(r, 4)
            if r >= RECALL_TARGET:
                ef, recall = e, r
                break
        if ef is None:
            ef, recall = EF_SWEEP[-1], sweep[EF_SWEEP[-1]]
        shape = None
        if path != "exact":
            # the launch shape for this batch (results do not depend on it)
            if args.fast_shape:
                shape = tuple(int(x) for x in args.fast_shape.split(","))
                idx.set_fast_params(*shape)
            else:
                shape, _ = idx.tune_fast(q_dev, k, ef, args.expand, stream)

        def per_query_counts():
            cnt = torch.zeros((nq, 6), dtype=torch.int32, device=dev)
            call(path, ef, counters=cnt)
            torch.cuda.synchronize()
            return cnt.double().sum(0).cpu().numpy() / nq

        c = per_query_counts()
        fetched = c[1] + c[4]
        if path != "exact":
            # the tuned walk forgets ids in its small recently-seen table and
            # fetches some rows again; a 32768-slot table forgets almost
            # none, so its count is the (near) unique rows the walk needs
            idx.set_fast_params(shape[0], 15, 1)
            c = per_query_counts()
            idx.set_fast_params(*shape)
        hops_u, dist_u, hops0, dist0 = c[0], c[1], c[3], c[4]
        # algorithmic bytes per query of the dominant kernel: the rows whose
        # distances it needs (traversal rows: f16 padded to 32 bytes, fp8 to
        # 16) and the adjacency lists it reads
        trav_bytes = {"exact": args.dim * 4, "f16": (args.dim * 2 + 31) // 32 * 32,
                      "fp8": (args.dim + 15) // 16 * 16}[path]
        adj_bytes = hops0 * 2 * args.M * 4 + hops_u * args.M * 4
        bpq = (dist_u + dist0) * trav_bytes + adj_bytes
        fetched_bpq = fetched * trav_bytes + adj_bytes
        for _ in range(args.warmup):
            call(path, ef)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        times, kernel_ms = [], []
        if path != "exact":
            idx.set_fast_timing(True)
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                flush.fill_(1)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                call(path, ef)
                b.record(stream)
                b.synchronize()
                times.append(a.elapsed_time(b))
                # the dominant kernel alone: the walk (events the library
                # records around it on this stream), or the exact search
                kernel_ms.append(idx.fast_timing()[0] if path != "exact" else times[-1])
        torch.cuda.synchronize()
        if path != "exact":
            idx.set_fast_timing(False)
        total_ms = float(sum(times))
        if world > 1:
            t = torch.tensor([total_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        # end to end through the C ABI with pinned host buffers
        for _ in range(args.warmup):
            host_call(path, ef)
        e2e = []
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            host_call(path, ef)
            e2e.append(time.perf_counter() - t0)
        e2e_s = float(sum(e2e))
        if world > 1:
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        ms = total_ms / args.steps
        return {"path": path, "ef": ef, "recall": recall, "sweep": sweep, "ms_per_step": ms, "shape": shape,
                "fetched_bytes_per_query": fetched_bpq, "rows_fetched": fetched,
                "kernel_ms": float(np.mean(kernel_ms)),
                "qps": world * nq * args.steps / (total_ms / 1e3), "e2e_qps": world * nq * args.steps / e2e_s,
                "bytes_per_query": bpq, "dist_evals": dist_u + dist0, "hops0": hops0, "hops_u": hops_u,
                "clocks": clk.summary()}

    results = {}
    for path in args.paths.split(","):
        results[path] = measure(path)
        log(args, f"[{rank}] {path}: ef={results[path]['ef']} recall={results[path]['recall']:.4f} "
                  f"qps={results[path]['qps']:.0f} e2e={results[path]['e2e_qps']:.0f}")
    ok = [r for r in results.values() if r["recall"] >= RECALL_TARGET] or list(results.values())
    best = max(ok, key=lambda r: r["qps"])
    peak, peak_kind = measured_peaks()
    kernel = "search_exact_kernel" if best["path"] == "exact" else "walk_kernel"
    achieved = best["bytes_per_query"] * nq / (best["kernel_ms"] / 1e3) / 1e9
    tr = ncu_traffic_per_query(kernel)
    traffic = None
    if (tr and tr.get("workload") == "1Mx96" and tr.get("path") == best["path"] and tr.get("ef") == best["ef"]
            and "dram_bytes_per_query" in tr):
        traffic = round(tr["dram_bytes_per_query"] * nq)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td:
            gp = os.path.join(td, "g.pkg")
            idx.save(gp)
            cpu = cpu_baseline(args, gp, queries, results.get("exact", best)["ef"])

    if rank == 0:
        plain = results.get("exact")
        line = {
            "metric": METRIC_NAME,
            "value": round(best["qps"], 1),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(best["ms_per_step"], 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded Gaussian mixture, unit rows; stands in for the public datasets)",
            "config": {"workload": f"{args.n // 1000}k x {args.dim} f32 IP, M={args.M}, efC={args.efc}, "
                                   f"{nq} queries per GPU, k={k}",
                       "n": args.n, "dim": args.dim, "metric": "ip", "M": args.M, "ef_construction": args.efc,
                       "queries_per_gpu": nq, "k": k, "path": best["path"], "ef": best["ef"],
                       "recall_at_10": round(best["recall"], 4),
                       "paths": {p: {"ef": r["ef"], "recall_at_10": round(r["recall"], 4), "qps": round(r["qps"], 1),
                                     "e2e_qps": round(r["e2e_qps"], 1), "ms_per_step": round(r["ms_per_step"], 4),
                                     "kernel_ms": round(r["kernel_ms"], 4), "launch_shape": r["shape"],
                                     "ef_sweep_recall": r["sweep"]} for p, r in results.items()},
                       "speedup_vs_plain_fp32": round(best["qps"] / plain["qps"], 3) if plain else None,
                       "l2": "flushed between steps (256 MiB write); index 640 MB > L2",
                       "build_s": round(build_s, 2), "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(best["e2e_qps"], 1), "unit": "queries/s",
                    "h2d_bytes_per_step": nq * args.dim * 4, "d2h_bytes_per_step": nq * k * 8},
            # exact: the search kernel; fast: query conversion, walk, re-rank
            "gpu_launches": args.steps * (1 if best["path"] == "exact" else 3),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                         "kernel": kernel, "kernel_ms": round(best["kernel_ms"], 4),
                         "bytes_per_query": round(best["bytes_per_query"], 1),
                         "fetched_bytes_per_query": round(best["fetched_bytes_per_query"], 1),
                         "per_query": {"dist_evals": round(best["dist_evals"], 1), "hops_l0": round(best["hops0"], 1),
                                       "hops_upper": round(best["hops_u"], 1),
                                       "rows_fetched": round(best["rows_fetched"], 1)}},
            "cpu_baseline": cpu,
            "clocks": best["clocks"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    """The reference's own Build and AnnSearch on the host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    from pickle_b200 import datasets
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pk_ref was not built"}))
        return
    base, queries = make_data(args, 0)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        gp = os.path.join(td, "ref.pkg")
        t0 = time.time()
        binfo = oracle.ref_build(base, "ip", args.M, args.efc, gp, threads=threads)
        build_s = time.time() - t0
        sample = queries[: args.cpu_sample]
        gt, _ = datasets.exact_knn(base, sample, args.k, "ip")
        ef, recall, sweep = EF_SWEEP[-1], None, {}
        for e in EF_SWEEP:
            ri, _, _ = oracle.ref_search(gp, sample, args.k, e, threads=threads)
            r = datasets.recall_at_k(ri, gt, args.k)
            sweep[e] = round(r, 4)
            if r >= RECALL_TARGET:
                ef, recall = e, r
                break
        steps = []
        for _ in range(args.warmup):
            oracle.ref_search(gp, sample, args.k, ef, threads=threads, want_results=False)
        for _ in range(args.steps):
            _, _, info = oracle.ref_search(gp, sample, args.k, ef, threads=threads, want_results=False)
            steps.append(info["median_s"])
    total = sum(steps)
    value = len(sample) * args.steps / total
    line = {
        "metric": METRIC_NAME, "value": round(value, 1), "unit": "queries/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic (seeded Gaussian mixture, unit rows)",
        "config": {"workload": f"{args.n // 1000}k x {args.dim} f32 IP, M={args.M}, efC={args.efc}, k={args.k}",
                   "ef": ef, "recall_at_10": recall, "ef_sweep_recall": sweep, "build_s": round(build_s, 1),
                   "queries_per_step": len(sample)},
        "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(sample)} queries per step, batch AnnSearch, graph built by the "
                                   f"reference's own Build on {threads} threads"},
        "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
