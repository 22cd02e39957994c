"""Python access to the oracle.  TEST INFRASTRUCTURE.

Two checkers live here:

* ``OraGraph`` wraps ``libpk_oracle.so``, the C restatement of the reference's
  HNSW search and insert path (pk_oracle.c).
* ``ref_build`` / ``ref_search`` / ``ref_dist`` run ``_ref/pk_ref``, the
  reference's own headers compiled around ref_harness.cpp, as a subprocess
  (one graph per process, as the reference requires).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this package, and only to check or to time the reference; the product in
``pickle_b200`` never imports it.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpk_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "pk_ref")

# DataType / DistFunc values of the reference (include/common.hpp:21-33)
DTYPES = {np.dtype(np.uint8): 0, np.dtype(np.int8): 1, np.dtype(np.float32): 2, np.dtype(np.float16): 3}
METRICS = {"l2": 1, "ip": 2}
GROWTH_REFERENCE, GROWTH_CAPPED = 0, 1

_lib = None


def build_oracle() -> None:
    """Compile libpk_oracle.so (and _ref/pk_ref where the reference is present)."""
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_oracle()
        L = ctypes.CDLL(LIB_PATH)
        P, I64, I32, F, VP = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float, ctypes.c_void_p
        L.ora_load.restype = P
        L.ora_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        L.ora_new.restype = P
        L.ora_new.argtypes = [I32, I32, I64, I64, I64, I64, VP, I32]
        L.ora_free.argtypes = [P]
        L.ora_save.argtypes = [P, ctypes.c_char_p]
        L.ora_info.argtypes = [P, VP]
        L.ora_insert.argtypes = [P, ctypes.c_int32, VP]
        L.ora_build.argtypes = [P, VP, VP, I64]
        L.ora_search.argtypes = [P, VP, I64, I32, I32, I32, VP, VP, VP]
        L.ora_distance.restype = F
        L.ora_distance.argtypes = [I32, I32, VP, VP, I64]
        L.ora_cumulative_probability.argtypes = [I64, VP, I32]
        L.ora_layer.argtypes = [P, I32] + [VP] * 7
        L.ora_set_float_order.argtypes = [I32]
        L.ora_search_fork.argtypes = [P, VP, I64, I32, I32, I32, I32, VP, VP, VP, I32, VP, VP, VP, VP, I64, VP]
        _lib = L
    return _lib


# Float summation orders (pk_oracle.h): the reference's source order, the
# device library's order, or distances looked up in a table.
ORDER_SOURCE, ORDER_DEVICE, ORDER_TABLE = 0, 1, 2


class float_order:
    """Context manager: float32 / float16 distances of the restatement in the
    given order (ORDER_SOURCE or ORDER_DEVICE) while it is active."""

    def __init__(self, order: int):
        self.order = order

    def __enter__(self):
        lib().ora_set_float_order(self.order)
        return self

    def __exit__(self, *exc):
        lib().ora_set_float_order(ORDER_SOURCE)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class OraGraph:
    """An HNSW graph held by the C restatement."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def load(cls, path: str) -> "OraGraph":
        rc = ctypes.c_int(0)
        h = lib().ora_load(path.encode(), ctypes.byref(rc))
        if not h:
            raise IOError(f"oracle could not load {path}: {rc.value}")
        return cls(h)

    @classmethod
    def new(cls, metric: str, dtype, dim: int, M: int, efc: int, levels: np.ndarray,
            growth: int = GROWTH_REFERENCE) -> "OraGraph":
        levels = np.ascontiguousarray(levels, dtype=np.uint8)
        h = lib().ora_new(METRICS[metric], DTYPES[np.dtype(dtype)], dim, M, efc, len(levels), _ptr(levels), growth)
        if not h:
            raise ValueError("bad oracle graph parameters")
        return cls(h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ora_free(self.h)
            self.h = None

    def info(self) -> dict:
        out = np.zeros(8, np.int64)
        err = lib().ora_info(self.h, _ptr(out))
        keys = ["n0", "num_layers", "enter_level", "capacity", "dim", "M", "metric", "dtype"]
        d = {k: int(v) for k, v in zip(keys, out)}
        d["err"] = err
        return d

    def build(self, data: np.ndarray, order: np.ndarray) -> None:
        data = np.ascontiguousarray(data)
        order = np.ascontiguousarray(order, dtype=np.int32)
        rc = lib().ora_build(self.h, _ptr(data), _ptr(order), len(order))
        if rc != 0:
            raise RuntimeError(f"oracle build failed: {rc}")

    def save(self, path: str) -> None:
        rc = lib().ora_save(self.h, path.encode())
        if rc != 0:
            raise IOError(f"oracle save failed: {rc}")

    def search(self, queries: np.ndarray, k: int, ef: int, threads: int = 0, counters: bool = False):
        q = np.ascontiguousarray(queries)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.float32)
        cnt = np.zeros((nq, 6), np.int64) if counters else None
        rc = lib().ora_search(self.h, _ptr(q), nq, k, ef, threads, _ptr(ids), _ptr(dists),
                              _ptr(cnt) if counters else None)
        if rc != 0:
            raise RuntimeError(f"oracle search failed: {rc}")
        return (ids, dists, cnt) if counters else (ids, dists)

    def search_fork(self, queries: np.ndarray, k: int, ef: int, order_a: int, order_b: int, table=None,
                    threads: int = 0, touched_cap: int = 0):
        """AnnSearch replayed with two sets of float distances (ora_search_fork).

        order_a drives the search; order_b (ORDER_SOURCE, ORDER_DEVICE, or
        ORDER_TABLE with table = (offsets[nq+1] int64, keys int32, values
        float32), keys sorted per query) is compared at every decision.
        Returns (ids, dists, fork, touched): fork is nq x 6 float64 =
        {forked, where, a_x, a_y, b_x, b_y} for the first comparison whose
        outcome differs (where: 1 SlideLayer, 2 early exit, 3 admission,
        4 heap order, 5 table miss); touched (with touched_cap > 0) is a list
        per query of the row keys (external id, -1 = zero row) whose
        distances the order_a search evaluated."""
        q = np.ascontiguousarray(queries)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.float32)
        fork = np.zeros((nq, 6), np.float64)
        toff = tkey = tval = None
        if order_b == ORDER_TABLE:
            toff, tkey, tval = (np.ascontiguousarray(table[0], np.int64), np.ascontiguousarray(table[1], np.int32),
                                np.ascontiguousarray(table[2], np.float32))
        touched = np.empty((nq, max(touched_cap, 1)), np.int32) if touched_cap else None
        tn = np.zeros(nq, np.int64)
        rc = lib().ora_search_fork(self.h, _ptr(q), nq, k, ef, order_a, order_b,
                                   _ptr(toff) if toff is not None else None, _ptr(tkey) if tkey is not None else None,
                                   _ptr(tval) if tval is not None else None, threads, _ptr(ids), _ptr(dists),
                                   _ptr(fork), _ptr(touched) if touched is not None else None, touched_cap, _ptr(tn))
        if rc != 0:
            raise RuntimeError(f"oracle fork search failed: {rc}")
        lists = None
        if touched is not None:
            if (tn > touched_cap).any():
                raise ValueError(f"touched_cap {touched_cap} < {int(tn.max())}")
            lists = [touched[i, :tn[i]].copy() for i in range(nq)]
        return ids, dists, fork, lists

    def layer(self, level: int) -> dict:
        n, cap = ctypes.c_int64(), ctypes.c_int64()
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        rc = lib().ora_layer(self.h, level, ctypes.byref(n), ctypes.byref(cap), *[ctypes.byref(p) for p in ptrs])
        if rc != 0:
            raise IndexError(level)
        n, cap = n.value, cap.value

        def arr(p, ctype, count, dt):
            return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctype)), shape=(count,)).astype(dt).copy()

        return {
            "n": n, "cap": cap,
            "ext": arr(ptrs[0], ctypes.c_int32, n, np.int32),
            "degree": arr(ptrs[1], ctypes.c_int16, n, np.int16),
            "heuristic": arr(ptrs[2], ctypes.c_int16, n, np.int16),
            "adj": arr(ptrs[3], ctypes.c_int32, n * cap, np.int32),
            "dist": arr(ptrs[4], ctypes.c_float, n * cap, np.float32),
        }


def distance(metric: str, a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    return float(lib().ora_distance(DTYPES[a.dtype], METRICS[metric], _ptr(a), _ptr(b), a.shape[-1]))


def cumulative_probability(M: int) -> np.ndarray:
    out = np.zeros(64, np.float64)
    n = lib().ora_cumulative_probability(M, _ptr(out), 64)
    return out[:n].copy()


# ---------------------------------------------------------------- reference ---

def ref_available() -> bool:
    return os.access(REF_BIN, os.X_OK)


def _run_ref(args, timeout=3600) -> dict:
    p = subprocess.run([REF_BIN] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"pk_ref {args[0]} failed ({p.returncode}): {p.stderr.strip()[-400:]}")
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    return json.loads(lines[-1]) if lines else {}


def ref_build(data: np.ndarray, metric: str, M: int, efc: int, out_path: str, threads: int = 0,
              order: np.ndarray | None = None, levels: np.ndarray | None = None) -> dict:
    """HNSWGraph::Build with the reference's code; writes a v2 graph file."""
    with tempfile.TemporaryDirectory() as td:
        dp = os.path.join(td, "data.npy")
        np.save(dp, np.ascontiguousarray(data))
        args = ["build", "--data", dp, "--metric", metric, "--M", M, "--efc", efc, "--out", out_path]
        if threads:
            args += ["--threads", threads]
        if order is not None:
            op = os.path.join(td, "order.npy")
            np.save(op, np.ascontiguousarray(order, dtype=np.int32))
            args += ["--order", op]
        if levels is not None:
            lp = os.path.join(td, "levels.npy")
            np.save(lp, np.ascontiguousarray(levels, dtype=np.uint8))
            args += ["--levels", lp]
        return _run_ref(args)


def ref_search(graph_path: str, queries: np.ndarray, k: int, ef: int, threads: int = 0, repeat: int = 1,
               metrics: bool = False, dynamic: bool = False, want_results: bool = True, k_per_query=None,
               ef_per_query=None):
    """Batch AnnSearch with the reference's code on a v2 graph file.  With
    k_per_query / ef_per_query, each query runs the single-query AnnSearch
    with its own values (k is then the width of the returned rows)."""
    with tempfile.TemporaryDirectory() as td:
        qp = os.path.join(td, "q.npy")
        np.save(qp, np.ascontiguousarray(queries))
        args = ["search", "--graph", graph_path, "--queries", qp, "--k", k, "--ef", ef, "--repeat", repeat]
        if k_per_query is not None:
            kp, ep = os.path.join(td, "kq.npy"), os.path.join(td, "efq.npy")
            np.save(kp, np.ascontiguousarray(k_per_query, np.int32))
            np.save(ep, np.ascontiguousarray(ef_per_query, np.int32))
            args += ["--kq", kp, "--efq", ep]
        if threads:
            args += ["--threads", threads]
        if metrics:
            args += ["--metrics"]
        if dynamic:
            args += ["--dynamic"]
        ip, dp = os.path.join(td, "ids.npy"), os.path.join(td, "d.npy")
        if want_results:
            args += ["--ids", ip, "--dists", dp]
        info = _run_ref(args)
        if want_results:
            return np.load(ip), np.load(dp), info
        return None, None, info


def ref_dist(metric: str, a: np.ndarray, b: np.ndarray, dynamic: bool = False) -> np.ndarray:
    """Row-wise pickle::Distance with the reference's code."""
    with tempfile.TemporaryDirectory() as td:
        ap, bp, op = (os.path.join(td, n) for n in ("a.npy", "b.npy", "o.npy"))
        np.save(ap, np.ascontiguousarray(a))
        np.save(bp, np.ascontiguousarray(b))
        args = ["dist", "--a", ap, "--b", bp, "--metric", metric, "--out", op]
        if dynamic:
            args += ["--dynamic"]
        _run_ref(args)
        return np.load(op)
