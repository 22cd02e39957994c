"""HNSW search throughput on one B200 (and N replicas), low-precision walk with
exact re-rank against the plain exact search.

Workload (default, the configuration the target is stated on): 10M base
vectors, dim 128, stored as float16, from a 1024-component Gaussian mixture
(unit-normal centres, sigma 0.5); L2; M = 32, ef_construction = 200, graph
built on the GPU; one batch of 100k queries from the same mixture, each with
its own k uniform in {1, 10, 100} and ef uniform in [max(k, 16), 512].  Seeded
synthetic stand-ins (the public datasets are not available offline).

A step is one search of the whole 100k-query batch.
  value   device-resident queries/s of the best path on the mixed batch: CUDA
          events around each search on its stream; the index (10.7 GB) is far
          larger than L2, and a 256 MiB buffer is written between steps.
  e2e     the same batch through the C ABI with host buffers
          (pk_index_search_fast_host_var / pk_index_search): pinned host
          queries and per-query k/ef in, ids and distances out, copies inside
          the timed region.
  config.paths  per path (exact = the drop-in search that replays the
          reference's heaps; f16 / fp8 = low-precision walk + exact re-rank):
          the mixed batch, and the recall@10 >= 0.95 point of a k = 10 ef
          sweep (recall on a 10k-query sample against float64 ground truth,
          QPS on the whole batch), each with its speed-up over the exact path.
  roofline  the walk kernel: algorithmic bytes per query (distinct traversal
          rows x their value bytes + adjacency rows read; the per-query work
          counters with a table large enough to forget nothing) x queries /
          the walk launches' device time (events the library records around
          them on the bench's stream), against the measured HBM bandwidth.
  cpu_baseline  the reference's own search (oracle/_ref/pk_ref, all host
          threads) on the same graph file, on a 2000-query sample of the
          mixed batch (its own k and ef per query).

--impl reference runs the reference's search on the host cores instead
(rank 0 only) on the same sample and prints the same line with impl =
reference.  Its graph is the GPU-built one (a reference Build of 10M rows
takes hours on the host); both arms share it through a file cache.

--workload c2 runs the earlier configuration instead: 1M x 96 float32 unit
rows (256-component mixture, sigma 0.3), inner product, M = 32, efC = 400,
10k queries, k = 10, and reports QPS at the smallest ef of a sweep with
recall@10 >= 0.95.

Multi-GPU (--gpus N; relaunches itself under torch.distributed.run when
WORLD_SIZE is unset): every rank holds a full replica and searches its own
batch; no collective is on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RECALL_TARGET = 0.95
WORKLOADS = {
    "c4": dict(n=10_000_000, nq=100_000, dim=128, dtype="f16", metric="l2", M=32, efc=200, mixed=True,
               sweep=[32, 48, 64, 80, 96, 112, 128, 160, 192, 256], sample=10_000),
    "c2": dict(n=1_000_000, nq=10_000, dim=96, dtype="f32", metric="ip", M=32, efc=400, mixed=False,
               sweep=[16, 24, 32, 36, 40, 44, 48, 56, 64, 80, 96, 112, 128, 160, 192, 256, 320, 384, 512],
               sample=10_000),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c4", choices=sorted(WORKLOADS))
    p.add_argument("--n", type=int, default=0, help="base rows (default: the workload's)")
    p.add_argument("--nq", type=int, default=0, help="queries per GPU (default: the workload's)")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-sample", type=int, default=2000, help="queries in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--verbose", action="store_true")
    p.add_argument("--paths", default="exact,f16,fp8", help="search paths to measure (exact, f16, fp8)")
    p.add_argument("--expand", type=int, default=1, help="entries expanded per step on the fast paths")
    p.add_argument("--fast-shape", default="", help="rows,filter_log2,warps for the fast walk instead of tuning")
    p.add_argument("--launch-check", action="store_true",
                   help="only start the ranks (gloo on the host), agree on the world size and exit")
    p.add_argument("--cache", default=os.environ.get("PK_BENCH_CACHE", os.path.join(tempfile.gettempdir(),
                                                                                   "pickle_b200_bench")),
                   help="directory for the built graph file, shared by both arms ('' = no cache)")
    return p.parse_args()


def log(args, *a):
    if args.verbose:
        print(*a, file=sys.stderr, flush=True)


def workload(args):
    w = dict(WORKLOADS[args.workload])
    if args.n:
        w["n"] = args.n
    if args.nq:
        w["nq"] = args.nq
    w["sample"] = min(w["sample"], w["nq"])
    return w


def workload_name(w):
    t = {"f16": "float16", "f32": "float32"}[w["dtype"]]
    s = f"{w['n'] // 1_000_000}M x {w['dim']} {t}, {w['metric'].upper()}, M={w['M']}, efC={w['efc']}, "
    if w["mixed"]:
        return s + f"{w['nq'] // 1000}k queries per GPU, k in {{1,10,100}}, ef in [max(k,16),512] per query"
    return s + f"{w['nq'] // 1000}k queries per GPU, k=10, smallest ef with recall@10>=0.95"


def metric_name(w):
    if w["mixed"]:
        return f"QPS of one {w['nq'] // 1000}k-query batch with per-query k and ef ({workload_name(w)})"
    return f"QPS at recall@10>=0.95 ({workload_name(w)})"


def make_data(w, seed, rank):
    from pickle_b200 import datasets
    if w["dtype"] == "f16":
        base, queries = datasets.gmm_f16(w["n"], w["nq"], w["dim"], ncomp=1024, sigma=0.5, seed=seed)
    else:
        base, queries = datasets.gmm_unit(w["n"], w["nq"], w["dim"], ncomp=256, sigma=0.3, seed=seed)
    if rank:
        queries = queries[np.random.default_rng(1000 + rank).permutation(len(queries))]
    return base, queries


def per_query_k_ef(w, nq, seed):
    """k uniform in {1, 10, 100}, ef uniform in [max(k, 16), 512] (mixed), else k = 10."""
    rng = np.random.default_rng(seed + 7)
    if not w["mixed"]:
        return np.full(nq, 10, np.int32), None
    kq = rng.choice([1, 10, 100], size=nq).astype(np.int32)
    efq = np.array([rng.integers(max(int(k), 16), 513) for k in kq], np.int32)
    return kq, efq


def recall_mixed(found, truth, ks):
    hit = 0
    for f, t, k in zip(found, truth, ks):
        hit += len(set(int(x) for x in f[:k] if x >= 0) & set(int(x) for x in t[:k]))
    return hit / float(np.sum(ks))


def lib_digest():
    from pickle_b200 import LIB_PATH
    h = hashlib.sha1()
    with open(LIB_PATH, "rb") as f:
        for blk in iter(lambda: f.read(1 << 22), b""):
            h.update(blk)
    return h.hexdigest()[:16]


def graph_file(args, w):
    if not args.cache:
        return None
    key = f"{args.workload}_{w['n']}_{w['dim']}_{args.seed}_{lib_digest()}"
    return os.path.join(args.cache, key + ".pkg")


def build_or_load(args, w, base, rank):
    """The GPU-built graph: loaded from the cache file when a run with the same
    workload, seed and library built it already, else built (and, on rank 0,
    saved).  Returns (index, build seconds or None, path of a saved copy or None)."""
    import torch

    from pickle_b200 import HNSWIndex
    path = graph_file(args, w)
    if path and os.path.exists(path):
        try:
            t0 = time.time()
            idx = HNSWIndex.load(path)
            log(args, f"[{rank}] loaded {path} in {time.time() - t0:.1f}s")
            return idx, None, path
        except Exception as e:  # a partial or stale file: build instead
            log(args, f"[{rank}] cache load failed ({e}); building")
    idx = HNSWIndex(w["dim"], base.dtype, w["metric"], M=w["M"], ef_construction=w["efc"])
    idx.set_seed(args.seed)
    torch.cuda.synchronize()
    t0 = time.time()
    idx.build(base)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    saved = None
    if path and rank == 0:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + f".tmp{os.getpid()}"
            idx.save(tmp)
            os.replace(tmp, path)
            saved = path
        except Exception as e:
            log(args, f"cache save failed: {e}")
    return idx, build_s, saved


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


def profiled_traffic(workload_key, path):
    """DRAM bytes per query of the walk from a committed ncu summary of the
    same workload and path (a figure of that capture, not of this run)."""
    try:
        with open(os.path.join(ROOT, "profiles", f"walk_kernel_{workload_key}_traffic.json")) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return None
    if "paths" in d:
        p = d["paths"].get(path)
        return dict(p, source=p.get("source", d.get("source"))) if p else None
    return d if d.get("path") == path else None


def cpu_reference(graph_path, queries, k, ef, kq, efq, repeat, warmup=0):
    """The reference's AnnSearch on a graph file, all host threads; returns
    (per-run seconds after the warm-up runs, threads)."""
    import oracle
    threads = os.cpu_count() or 1
    _, _, info = oracle.ref_search(graph_path, queries, k, ef, threads=threads, repeat=warmup + repeat,
                                   want_results=False, k_per_query=kq, ef_per_query=efq)
    return info["all_s"][warmup:], threads


def relaunch_distributed(args):
    """--gpus N without a torch.distributed environment: rerun this command
    under torch.distributed.run with N processes on this node."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


# -------------------------------------------------------------------- ours --

def run_ours(args):
    import ctypes

    import torch
    import torch.distributed as dist

    from pickle_b200 import datasets, lib
    from pickle_b200.groundtruth import gpu_knn

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE is {world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=30), device_id=dev)

    w = workload(args)
    base, queries = make_data(w, args.seed, rank)
    nq = len(queries)
    log(args, f"[{rank}] data ready")
    idx, build_s, saved = build_or_load(args, w, base, rank)
    log(args, f"[{rank}] index ready (build {build_s})")
    kq, efq = per_query_k_ef(w, nq, args.seed)
    kmax = int(kq.max())
    ns = w["sample"]
    gt = gpu_knn(base, queries[:ns], max(kmax, 10), w["metric"], dev)
    del base

    q_dev = torch.from_numpy(queries).to(dev)
    kq_dev = torch.from_numpy(kq).to(dev)
    efq_dev = torch.from_numpy(efq).to(dev) if efq is not None else None
    ids = torch.empty((nq, kmax), dtype=torch.int32, device=dev)
    ds = torch.empty((nq, kmax), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MiB > 126 MB of L2
    L = lib()

    def call(path, k, ef, mixed, counters=None, q=q_dev, out_i=ids, out_d=ds):
        kk = kq_dev[:q.shape[0]] if mixed else None
        ee = efq_dev[:q.shape[0]] if mixed else None
        if path == "exact":
            idx.search_device(q, k, ef, out_i, out_d, k_per_query=kk, ef_per_query=ee, counters=counters,
                              stream=stream)
        else:
            idx.search_fast_device(q, k, ef, out_i, out_d, k_per_query=kk, ef_per_query=ee, counters=counters,
                                   expand=args.expand, stream=stream)

    def timed(path, k, ef, mixed):
        """K timed steps (after W warm-up steps): total ms and per-step walk ms."""
        for _ in range(args.warmup):
            call(path, k, ef, mixed)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        times, kernel_ms = [], []
        if path != "exact":
            idx.set_fast_timing(True)
        # an NVTX range around the timed steps, for profilers to select
        torch.cuda.nvtx.range_push(f"timed {path} {'mixed' if mixed else 'k10'}")
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                flush.fill_(1)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                call(path, k, ef, mixed)
                b.record(stream)
                b.synchronize()
                times.append(a.elapsed_time(b))
                kernel_ms.append(idx.fast_timing()[0] if path != "exact" else times[-1])
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if path != "exact":
            idx.set_fast_timing(False)
        total = float(sum(times))
        if world > 1:
            t = torch.tensor([total], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total = float(t.item())
        return total, float(np.mean(kernel_ms)), clk.summary()

    def tune(path, k, ef, mixed):
        """The walk's launch shape: one for a uniform batch, one per list-width
        class for the mixed batch (returned as {class: shape})."""
        if path == "exact":
            return None
        if args.fast_shape:
            shape = tuple(int(x) for x in args.fast_shape.split(","))
            idx.set_fast_params(*shape)
            return shape
        nt = min(nq, 20_000)
        if mixed:
            # per list width (each class alone at its widest ef), then the
            # candidates - those shapes, and a few shapes for every width -
            # timed on the batch itself, where the widths run side by side
            per = idx.tune_fast_classes(q_dev[:nt // 2], k, ef, args.expand, stream)
            cands = [{c: v[0] for c, v in per.items()}] + [(32, hl, wp) for hl in (8, 10) for wp in (1, 2, 4)]
            best = None
            for cand in cands:
                apply_shape(cand)
                ms = []
                for _ in range(3):
                    flush.fill_(2)
                    a = torch.cuda.Event(enable_timing=True)
                    b = torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    call(path, k, ef, True)
                    b.record(stream)
                    b.synchronize()
                    ms.append(a.elapsed_time(b))
                t = min(ms[1:])
                if best is None or t < best[0]:
                    best = (t, cand)
            apply_shape(best[1])
            return best[1]
        shape, _ = idx.tune_fast(q_dev[:nt], k, ef, args.expand, stream)
        return shape

    def apply_shape(shape):
        if isinstance(shape, dict):
            idx.set_fast_params(0, 0, 0)
            for c, sh in shape.items():
                idx.set_fast_class_params(c, *sh)
        elif shape is not None:
            idx.set_fast_params(*shape)

    def counts(path, k, ef, mixed, shape):
        """Per-query means of the six work counters; for the fast paths with a
        32768-slot recently-seen table, which forgets almost nothing, so that
        the rows counted are the (near) distinct rows the walk needs, and with
        the tuned table (the rows it actually fetches)."""
        cnt = torch.zeros((nq, 6), dtype=torch.int32, device=dev)
        call(path, k, ef, mixed, counters=cnt)
        torch.cuda.synchronize()
        fetched = cnt.double().mean(0).cpu().numpy()
        if path == "exact":
            return fetched, fetched
        idx.set_fast_params(16, 15, 1)
        cnt.zero_()
        call(path, k, ef, mixed, counters=cnt)
        torch.cuda.synchronize()
        apply_shape(shape)
        return cnt.double().mean(0).cpu().numpy(), fetched

    elem = {"f16": 2, "f32": 4}[w["dtype"]]
    trav_bytes = {"exact": w["dim"] * elem, "f16": (w["dim"] * 2 + 31) // 32 * 32,
                  "fp8": (w["dim"] + 31) // 32 * 32}

    def algorithmic_bytes(path, c):
        # distinct rows x their value bytes + the adjacency rows read (layer 0
        # holds 2M slots per node, upper layers M)
        return (c[1] + c[4]) * trav_bytes[path] + c[3] * 2 * w["M"] * 4 + c[0] * w["M"] * 4

    results = {}
    for path in args.paths.split(","):
        if path != "exact":
            idx.prepare_fast(path)
        r = {"path": path}
        # the k = 10 recall@10 >= 0.95 point: recall on the sample, QPS on the whole batch
        sweep, ef10 = {}, None
        qs = q_dev[:ns]
        ids10 = torch.empty((ns, 10), dtype=torch.int32, device=dev)
        ds10 = torch.empty((ns, 10), dtype=torch.float32, device=dev)
        for e in w["sweep"]:
            call(path, 10, e, False, q=qs, out_i=ids10, out_d=ds10)
            torch.cuda.synchronize()
            rc = datasets.recall_at_k(ids10.cpu().numpy(), gt, 10)
            sweep[e] = round(rc, 4)
            if rc >= RECALL_TARGET:
                ef10 = e
                break
        if ef10 is None:
            ef10 = w["sweep"][-1]
        shape10 = tune(path, 10, ef10, False)
        tot10, kms10, clk10 = timed(path, 10, ef10, False)
        r["k10"] = {"ef": ef10, "recall_at_10": sweep[ef10], "ef_sweep_recall": sweep, "launch_shape": shape10,
                    "qps": world * nq * args.steps / (tot10 / 1e3), "ms_per_step": tot10 / args.steps,
                    "kernel_ms": kms10, "clocks": clk10}
        if w["mixed"]:
            efmax = int(efq.max())
            shape = tune(path, kmax, efmax, True)
            tot, kms, clk = timed(path, kmax, efmax, True)
            call(path, kmax, efmax, True)
            torch.cuda.synchronize()
            rec = recall_mixed(ids[:ns].cpu().numpy(), gt, kq[:ns])
            c_alg, c_fetch = counts(path, kmax, efmax, True, shape)
            r["mixed"] = {"recall_at_k": rec, "launch_shape": shape, "qps": world * nq * args.steps / (tot / 1e3),
                          "ms_per_step": tot / args.steps, "kernel_ms": kms, "clocks": clk,
                          "bytes_per_query": algorithmic_bytes(path, c_alg), "counters": c_alg.tolist(),
                          "rows_fetched": float(c_fetch[1] + c_fetch[4])}
        else:
            c_alg, c_fetch = counts(path, 10, ef10, False, shape10)
            r["k10"].update(bytes_per_query=algorithmic_bytes(path, c_alg), counters=c_alg.tolist(),
                            rows_fetched=float(c_fetch[1] + c_fetch[4]))
        results[path] = r
        log(args, f"[{rank}] {path}: " + json.dumps({x: {kk: v for kk, v in r[x].items() if kk != 'clocks'}
                                                     for x in ("k10", "mixed") if x in r}))

    head = "mixed" if w["mixed"] else "k10"
    ok = [r for r in results.values() if w["mixed"] or r["k10"]["recall_at_10"] >= RECALL_TARGET]
    best = max(ok or list(results.values()), key=lambda r: r[head]["qps"])
    bp = best["path"]
    bh = best[head]

    # end to end through the C ABI with pinned host buffers
    qh = torch.from_numpy(queries).pin_memory()
    kh = torch.from_numpy(kq).pin_memory()
    eh = torch.from_numpy(efq if efq is not None else np.full(nq, bh.get("ef", best["k10"]["ef"]), np.int32))
    eh = eh.pin_memory()
    stride = kmax if w["mixed"] else 10
    ih = torch.empty((nq, stride), dtype=torch.int32).pin_memory()
    dh = torch.empty((nq, stride), dtype=torch.float32).pin_memory()
    ef_u = best["k10"]["ef"]
    if bp != "exact":
        apply_shape(bh["launch_shape"])

    def host_call():
        qp, ip_, dp = (ctypes.c_void_p(t.data_ptr()) for t in (qh, ih, dh))
        if w["mixed"] and bp != "exact":
            rc = L.pk_index_search_fast_host_var(idx._h, qp, nq, ctypes.c_void_p(kh.data_ptr()),
                                                 ctypes.c_void_p(eh.data_ptr()), stride, ip_, dp, args.expand)
        elif w["mixed"]:
            rc = L.pk_index_search_var(idx._h, qp, nq, ctypes.c_void_p(kh.data_ptr()), ctypes.c_void_p(eh.data_ptr()),
                                       stride, ip_, dp)
        elif bp == "exact":
            rc = L.pk_index_search(idx._h, qp, nq, stride, ef_u, ip_, dp)
        else:
            rc = L.pk_index_search_fast_host(idx._h, qp, nq, stride, ef_u, ip_, dp, args.expand)
        if rc != 0:
            raise RuntimeError(L.pk_last_error().decode())

    for _ in range(args.warmup):
        host_call()
    e2e = []
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        host_call()
        e2e.append(time.perf_counter() - t0)
    e2e_s = float(sum(e2e))
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_qps = world * nq * args.steps / e2e_s

    peak, peak_kind = measured_peaks()
    kernel = "search_exact_kernel" if bp == "exact" else "walk_kernel"
    rf = best["mixed"] if w["mixed"] else best["k10"]
    achieved = rf["bytes_per_query"] * nq / (rf["kernel_ms"] / 1e3) / 1e9
    tr = profiled_traffic(args.workload, bp)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            gp = saved or graph_file(args, w)
            tmpdir = None
            if not gp or not os.path.exists(gp):
                tmpdir = tempfile.mkdtemp(prefix="pk_bench_")
                gp = os.path.join(tmpdir, "g.pkg")
                idx.save(gp)
            ns_cpu = min(args.cpu_sample, nq)
            if w["mixed"]:
                secs, threads = cpu_reference(gp, queries[:ns_cpu], kmax, int(efq.max()), kq[:ns_cpu],
                                              efq[:ns_cpu], 3)
                what = f"{ns_cpu} queries of the mixed batch with their own k and ef"
            else:
                secs, threads = cpu_reference(gp, queries[:ns_cpu], 10, best["k10"]["ef"], None, None, 3)
                what = f"{ns_cpu} of the {nq} queries at ef={best['k10']['ef']}"
            cpu = {"value": round(ns_cpu / statistics.median(secs), 1), "unit": "queries/s", "cores": threads,
                   "kind": "reference",
                   "sample": what + ", same graph file, median of 3 batch runs (steady clock around the batch)"}
            if tmpdir:
                os.remove(gp)
                os.rmdir(tmpdir)

    if rank == 0:
        plain = results.get("exact")

        def path_line(r):
            out = {}
            for key in ("mixed", "k10"):
                if key not in r:
                    continue
                x = r[key]
                out[key] = {kk: (round(v, 4) if isinstance(v, float) else v) for kk, v in x.items()
                            if kk not in ("clocks", "counters")}
                if plain and key in plain:
                    out[key]["speedup_vs_plain_fp32"] = round(x["qps"] / plain[key]["qps"], 3)
            return out

        launches = 1 if bp == "exact" else (3 + (8 if w["mixed"] else 1))
        line = {
            "metric": metric_name(w),
            "value": round(bh["qps"], 1),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(bh["ms_per_step"], 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f16" if w["dtype"] == "f16" else "f32",
            "data": "synthetic (seeded Gaussian mixture; stands in for the public datasets)",
            "config": {"workload": workload_name(w), "n": w["n"], "dim": w["dim"], "metric": w["metric"],
                       "M": w["M"], "ef_construction": w["efc"], "queries_per_gpu": nq, "path": bp,
                       "recall": round(bh.get("recall_at_k", bh.get("recall_at_10", 0.0)), 4),
                       "recall_sample": f"first {ns} queries, float64 exact ground truth",
                       "paths": {p: path_line(r) for p, r in results.items()},
                       "speedup_vs_plain_fp32": (round(bh["qps"] / plain[head]["qps"], 3) if plain else None),
                       "l2": "index 10.7 GB >> L2; 256 MiB written between steps" if w["mixed"] else
                             "index > L2; 256 MiB written between steps",
                       "graph": ("GPU build " + (f"{build_s:.1f} s" if build_s is not None else
                                                 "loaded from the bench's graph cache")),
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e_qps, 1), "unit": "queries/s",
                    "h2d_bytes_per_step": int(queries.nbytes + (kq.nbytes + efq.nbytes if w["mixed"] else 0)),
                    "d2h_bytes_per_step": int(nq * stride * 8)},
            "gpu_launches": args.steps * launches,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": (round(tr["dram_bytes_per_query"] * nq) if tr else None),
                         "traffic_source": (tr["source"] if tr else None),
                         "kernel": kernel, "kernel_ms": round(rf["kernel_ms"], 4),
                         "bytes_per_query": round(rf["bytes_per_query"], 1),
                         "rows_fetched_per_query": round(rf["rows_fetched"], 1),
                         "per_query": dict(zip(["hops_upper", "dists_upper", "nbrs_upper", "hops_l0", "dists_l0",
                                                "nbrs_l0"], [round(v, 1) for v in rf["counters"]]))},
            "cpu_baseline": cpu,
            "clocks": bh["clocks"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# --------------------------------------------------------------- reference --

def run_reference(args):
    """The reference's own AnnSearch (oracle/_ref/pk_ref) on the host cores,
    rank 0 only, on a sample of the same batch and the same GPU-built graph."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pk_ref was not built"}))
        return
    import torch

    from pickle_b200 import datasets
    from pickle_b200.groundtruth import gpu_knn
    w = workload(args)
    base, queries = make_data(w, args.seed, 0)
    idx, build_s, saved = build_or_load(args, w, base, 0)
    gp = saved or graph_file(args, w)
    tmpdir = None
    if not gp or not os.path.exists(gp):
        tmpdir = tempfile.mkdtemp(prefix="pk_bench_ref_")
        gp = os.path.join(tmpdir, "g.pkg")
        idx.save(gp)
    idx.close()
    ns = min(args.cpu_sample, len(queries))
    kq, efq = per_query_k_ef(w, len(queries), args.seed)
    sample = queries[:ns]
    gt = gpu_knn(base, sample, 100 if w["mixed"] else 10, w["metric"], torch.device("cuda"))
    del base
    threads = os.cpu_count() or 1
    # the k = 10 recall@10 >= 0.95 point of the reference on this graph
    sweep, ef10 = {}, w["sweep"][-1]
    for e in w["sweep"]:
        ri, _, _ = oracle.ref_search(gp, sample, 10, e, threads=threads)
        r = datasets.recall_at_k(ri, gt, 10)
        sweep[e] = round(r, 4)
        if r >= RECALL_TARGET:
            ef10 = e
            break
    if w["mixed"]:
        ri, _, info = oracle.ref_search(gp, sample, int(kq.max()), int(efq.max()), threads=threads,
                                        repeat=args.warmup + args.steps, k_per_query=kq[:ns],
                                        ef_per_query=efq[:ns])
        recall = recall_mixed(ri, gt, kq[:ns])
    else:
        ri, _, info = oracle.ref_search(gp, sample, 10, ef10, threads=threads, repeat=args.warmup + args.steps)
        recall = datasets.recall_at_k(ri, gt, 10)
    secs = info["all_s"][args.warmup:]
    total = float(sum(secs))
    value = ns * args.steps / total
    _, _, i10 = oracle.ref_search(gp, sample, 10, ef10, threads=threads, repeat=3, want_results=False)
    if tmpdir:
        os.remove(gp)
        os.rmdir(tmpdir)
    line = {
        "metric": metric_name(w), "value": round(value, 1), "unit": "queries/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16" if w["dtype"] == "f16" else "f32",
        "impl": "reference", "data": "synthetic (seeded Gaussian mixture)",
        "config": {"workload": workload_name(w), "queries_per_step": ns,
                   "recall": round(recall, 4), "k10": {"ef": ef10, "recall_at_10": sweep[ef10],
                                                       "ef_sweep_recall": sweep, "qps": round(i10["qps"], 1)},
                   "graph": "the GPU-built graph (a reference Build of this size takes hours on the host cores), "
                            + ("built here" if build_s is not None else "from the bench's graph cache")},
        "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": f"{ns} queries per step (the first {ns} of the batch"
                                   + (", each with its own k and ef)" if w["mixed"] else ")")
                                   + ", the reference's batch AnnSearch loop on all host threads"},
        "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def launch_check(args):
    """The process plumbing alone: every rank joins a gloo group, the world
    size is checked against --gpus and agreed by an all-reduce."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE is {world}")
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=60))
        t = torch.tensor([1.0])
        dist.all_reduce(t)
        seen = int(t.item())
        dist.destroy_process_group()
    else:
        seen = 1
    if rank == 0:
        print(json.dumps({"launch_check": True, "world": world, "ranks_joined": seen}), flush=True)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_distributed(args))
    if args.launch_check:
        launch_check(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
