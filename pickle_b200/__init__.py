"""pickle_b200: a B200 HNSW index (query and insert path) behind a C ABI.

The native library ``libpickle_b200.so`` (built by ``python -m pickle_b200.build``)
holds the whole index on the GPU and exports the entry points declared in
``include/pickle_b200.h``.  This module binds them with ctypes and offers
``HNSWIndex``, whose method names follow the reference's (broken) Python
binding (pybind/hnsw.cpp:116-128: build / search / save / load) and whose
semantics follow pickle::v2::HNSWGraph (include/hnsw.hpp:23-220).

There is no CPU implementation here: if the library is missing or no GPU is
present, every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["HNSWIndex", "Server", "PickleError", "lib", "DTYPES", "METRICS", "LIB_PATH"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpickle_b200.so")

# DataType and DistFunc values of the reference (include/common.hpp:21-33)
DTYPES = {np.dtype(np.uint8): 0, np.dtype(np.int8): 1, np.dtype(np.float32): 2, np.dtype(np.float16): 3}
NP_OF = {v: k for k, v in DTYPES.items()}
METRICS = {"l2": 1, "ip": 2}

ERRORS = {
    -1: "bad argument", -2: "out of memory", -3: "I/O error", -4: "bad graph file", -5: "CUDA error",
    -6: "invalid state", -7: "device wait timed out", -8: "scratch overflow", -9: "no CUDA device",
    -10: "capacity exceeded",
}


class PickleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m pickle_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, I64, I32, VP = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p
        PP = ctypes.POINTER(ctypes.c_void_p)
        L.pk_last_error.restype = ctypes.c_char_p
        L.pk_version.restype = ctypes.c_int
        L.pk_index_create.argtypes = [PP, ctypes.c_int, ctypes.c_int, I64, I64, I64]
        L.pk_index_destroy.argtypes = [P]
        L.pk_index_set_seed.argtypes = [P, ctypes.c_uint64]
        L.pk_index_set_levels.argtypes = [P, VP, I64]
        L.pk_index_build.argtypes = [P, VP, I64, VP, I32]
        L.pk_index_add.argtypes = [P, VP, I64, VP, I32]
        L.pk_index_search.argtypes = [P, VP, I64, I32, I32, VP, VP]
        L.pk_index_search_device.argtypes = [P, VP, I64, I32, I32, VP, VP, I32, VP, VP, VP, VP]
        L.pk_index_save.argtypes = [P, ctypes.c_char_p]
        L.pk_index_load.argtypes = [PP, ctypes.c_char_p]
        L.pk_index_info.argtypes = [P, VP]
        L.pk_index_layer.argtypes = [P, ctypes.c_int] + [VP] * 3 + [VP] * 6
        L.pk_index_prepare_fast.argtypes = [P, ctypes.c_int]
        L.pk_index_search_fast.argtypes = [P, VP, I64, I32, I32, VP, VP, I32, VP, VP, VP, I32, VP]
        L.pk_index_search_fast_host.argtypes = [P, VP, I64, I32, I32, VP, VP, I32]
        L.pk_index_set_fast_params.argtypes = [P, I32, I32, I32]
        L.pk_index_set_fast_timing.argtypes = [P, ctypes.c_int]
        L.pk_index_set_fast_visited.argtypes = [P, I32]
        L.pk_index_set_fast_merge.argtypes = [P, I32]
        L.pk_index_set_build_walk.argtypes = [P, I64]
        L.pk_index_fast_timing.argtypes = [P, VP, VP]
        L.pk_index_tune_fast.argtypes = [P, VP, I64, I32, I32, I32, VP, VP, VP]
        L.pk_index_tune_fast_classes.argtypes = [P, VP, I64, I32, I32, I32, VP, VP, VP]
        L.pk_index_set_fast_class_params.argtypes = [P, I32, I32, I32, I32]
        L.pk_index_search_noalloc.argtypes = [P, VP, I64, I32, I32, VP, VP, VP]
        L.pk_index_search_var.argtypes = [P, VP, I64, VP, VP, I32, VP, VP]
        L.pk_index_search_fast_host_var.argtypes = [P, VP, I64, VP, VP, I32, VP, VP, I32]
        L.pk_server_create.argtypes = [PP, P, ctypes.c_int, ctypes.c_int, I32, I32, I32, I32]
        L.pk_server_submit.argtypes = [P, VP, I32, I32, I32, ctypes.POINTER(ctypes.c_int64)]
        L.pk_server_wait.argtypes = [P, ctypes.c_int64, VP, VP, ctypes.POINTER(ctypes.c_double), I32]
        L.pk_server_stats.argtypes = [P, VP]
        L.pk_server_set_watchdog.argtypes = [P, ctypes.c_double]
        L.pk_server_destroy.argtypes = [P]
        L.pk_server_replay.argtypes = [P, VP, I64, VP, VP, VP, VP, VP, VP, I32, VP]
        L.pk_server_create_with_memory.argtypes = [PP, P, ctypes.c_int, ctypes.c_int, I32, I32, I32, I32, I64]
        L.pk_server_memory.argtypes = [P, VP]
        L.pk_server_request_bytes.argtypes = [P, I32, I32, I32, ctypes.POINTER(ctypes.c_int64)]
        for name in ["pk_index_create", "pk_index_destroy", "pk_index_set_seed", "pk_index_set_levels",
                     "pk_index_build", "pk_index_add", "pk_index_search", "pk_index_search_device",
                     "pk_index_save", "pk_index_load", "pk_index_info", "pk_index_layer", "pk_index_prepare_fast",
                     "pk_index_search_fast", "pk_index_search_fast_host", "pk_index_search_noalloc",
                     "pk_index_search_var", "pk_index_search_fast_host_var", "pk_index_tune_fast_classes",
                     "pk_index_set_fast_class_params",
                     "pk_server_create", "pk_server_submit", "pk_server_wait", "pk_server_stats",
                     "pk_server_set_watchdog", "pk_server_destroy", "pk_server_replay",
                     "pk_server_create_with_memory", "pk_server_memory", "pk_server_request_bytes"]:
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise PickleError(rc, lib().pk_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dev_ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class _class_or_instance:
    """A method that works on the class (returning a new object) and on an
    instance (acting on it), as HNSWIndex.load does."""

    def __init__(self, fn):
        self.fn = fn

    def __get__(self, obj, owner):
        def bound(*a, **kw):
            return self.fn(owner, obj, *a, **kw)
        bound.__doc__ = self.fn.__doc__
        return bound


class HNSWIndex:
    """An HNSW index resident in GPU memory.

    Two ways to make one:
      HNSWIndex(dim, dtype, metric="l2", M=32, ef_construction=100) mirrors
        HNSWGraph(max_degree, build_ef, DistFunc) (include/hnsw.hpp:27-36): the
        index exists at once, empty.
      HNSWIndex() mirrors the reference's Python binding (pybind/hnsw.cpp:
        116-127): set the properties search_ef (100), build_ef (100), top_k
        (10), M (32) and metric, then build(data) creates the index with the
        data's dimension and type (a later build(data) replaces it, as there).
    search(queries) uses top_k and search_ef and returns the ids, nq x top_k;
    search(queries, k, ef) returns (ids, distances).
    """

    def __init__(self, dim: int = 0, dtype=np.float32, metric: str = "l2", M: int = 32,
                 ef_construction: int = 100, _handle=None):
        self._h = None
        self._deferred = False
        self.search_ef = 100
        self.top_k = 10
        self.metric = metric
        self._M = M
        self._build_ef = ef_construction
        if _handle is not None:
            self._adopt(_handle)
        elif dim > 0:
            h = ctypes.c_void_p()
            _check(lib().pk_index_create(ctypes.byref(h), METRICS[metric], DTYPES[np.dtype(dtype)], dim, M,
                                         ef_construction))
            self._adopt(h)
        else:
            # the reference binding's default constructor: created by build()
            self._deferred = True
            self.dim = 0
            self.dtype = None

    def _adopt(self, h) -> None:
        self.close()
        self._h = h
        info = self.info()
        self.dim = info["dim"]
        self.dtype = NP_OF[info["dtype"]]
        self.metric = {1: "l2", 2: "ip"}[info["metric"]]
        self._M = info["M"]
        self._build_ef = info["ef_construction"]

    # ---- the reference binding's properties (pybind/hnsw.cpp:118-123) ----
    @property
    def M(self) -> int:
        return self._M

    @M.setter
    def M(self, value: int) -> None:
        if self._h is not None and not self._deferred:
            raise ValueError("M is fixed once the index exists (it was given to the constructor)")
        self._M = int(value)

    @property
    def build_ef(self) -> int:
        return self._build_ef

    @build_ef.setter
    def build_ef(self, value: int) -> None:
        if self._h is not None and not self._deferred:
            raise ValueError("build_ef is fixed once the index exists (it was given to the constructor)")
        self._build_ef = int(value)

    @property
    def ef_construction(self) -> int:
        return self._build_ef

    @property
    def num_layer(self) -> int:
        """Layers of the graph (0 before a build).  The reference binding binds
        this name to its top_k getter by mistake (pybind/hnsw.cpp:123); here it
        is the layer count its getNumLayer computes (:46)."""
        return self.info()["num_layers"] if self._h is not None else 0

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the module's globals may be gone
            pass

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pk_index_destroy(self._h)
            self._h = None

    # ---- construction -------------------------------------------------
    def set_seed(self, seed: int) -> None:
        _check(lib().pk_index_set_seed(self._h, seed))

    def set_levels(self, levels: np.ndarray) -> None:
        lv = np.ascontiguousarray(levels, dtype=np.uint8)
        _check(lib().pk_index_set_levels(self._h, _ptr(lv), len(lv)))

    def build(self, data: np.ndarray, ext_ids: np.ndarray | None = None, max_batch: int = 0) -> None:
        """HNSWGraph::Build: insert data[ext_ids[i]] with id ext_ids[i], i = 0..n-1
        (ext_ids None: 0..n-1).  On a default-constructed index this first
        creates the index from the data's shape and type and the M, build_ef
        and metric properties, replacing any earlier one."""
        if self._deferred:
            data = np.ascontiguousarray(data)
            if data.ndim != 2 or data.dtype not in DTYPES:
                raise ValueError("build expects a 2-D uint8, int8, float16 or float32 array")
            h = ctypes.c_void_p()
            _check(lib().pk_index_create(ctypes.byref(h), METRICS[self.metric], DTYPES[data.dtype], data.shape[1],
                                         self._M, self._build_ef))
            self.close()
            self._h = h
            self.dim = data.shape[1]
            self.dtype = data.dtype
        data = self._rows(data)
        ids = None if ext_ids is None else np.ascontiguousarray(ext_ids, dtype=np.int32)
        _check(lib().pk_index_build(self._h, _ptr(data), data.shape[0], _ptr(ids) if ids is not None else None,
                                    max_batch))

    def add(self, rows: np.ndarray, ext_ids: np.ndarray, max_batch: int = 0) -> None:
        """HNSWGraph::Insert for a batch of new rows."""
        rows = self._rows(rows)
        ids = np.ascontiguousarray(ext_ids, dtype=np.int32)
        if len(ids) != rows.shape[0]:
            raise ValueError("one external id per row")
        _check(lib().pk_index_add(self._h, _ptr(rows), rows.shape[0], _ptr(ids), max_batch))

    # ---- queries --------------------------------------------------------
    def search(self, queries: np.ndarray, k: int | None = None, ef: int | None = None):
        """HNSWGraph::AnnSearch(k, ef, queries).  With k and ef: (ids, dists),
        each nq x k, ascending.  Without them: the reference binding's
        search(query) (pybind/hnsw.cpp:73-101), k = top_k and ef = search_ef,
        returning the ids only."""
        q = self._rows(queries)
        nq = q.shape[0]
        kk = self.top_k if k is None else k
        ee = self.search_ef if ef is None else ef
        ids = np.empty((nq, kk), np.int32)
        dists = np.empty((nq, kk), np.float32)
        _check(lib().pk_index_search(self._h, _ptr(q), nq, kk, ee, _ptr(ids), _ptr(dists)))
        if k is None and ef is None:
            return ids
        return ids, dists

    def search_var(self, queries: np.ndarray, k_per_query: np.ndarray, ef_per_query: np.ndarray):
        """AnnSearch with a k and an ef per query (host buffers): (ids, dists),
        nq x max(k); row i holds k_per_query[i] results, then -1 / FLT_MAX."""
        q = self._rows(queries)
        kq = np.ascontiguousarray(k_per_query, np.int32)
        eq = np.ascontiguousarray(ef_per_query, np.int32)
        if len(kq) != q.shape[0] or len(eq) != q.shape[0]:
            raise ValueError("one k and one ef per query")
        stride = int(kq.max()) if len(kq) else 1
        ids = np.empty((q.shape[0], stride), np.int32)
        dists = np.empty((q.shape[0], stride), np.float32)
        _check(lib().pk_index_search_var(self._h, _ptr(q), q.shape[0], _ptr(kq), _ptr(eq), stride, _ptr(ids),
                                         _ptr(dists)))
        return ids, dists

    def search_device(self, queries, k: int, ef: int, out_ids, out_dists, k_per_query=None, ef_per_query=None,
                      counters=None, stream=None) -> None:
        """Device-resident search on torch CUDA tensors (asynchronous on `stream`).

        queries: (nq, dim) contiguous; out_ids int32 / out_dists float32: (nq, stride);
        k_per_query / ef_per_query: optional int32 (nq,); counters: optional int32 (nq, 6).
        """
        nq = queries.shape[0]
        stride = out_ids.shape[1]
        s = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _check(lib().pk_index_search_device(self._h, _dev_ptr(queries), nq, k, ef, _dev_ptr(k_per_query),
                                            _dev_ptr(ef_per_query), stride, _dev_ptr(out_ids), _dev_ptr(out_dists),
                                            _dev_ptr(counters), s))

    # ---- batched low-precision search ----------------------------------
    TRAVERSAL = {"f16": 1, "fp8": 2}

    def prepare_fast(self, traversal: str = "fp8") -> None:
        """Build the FP16 / FP8 (per-dimension scaled) copy the fast search walks with."""
        _check(lib().pk_index_prepare_fast(self._h, self.TRAVERSAL[traversal]))

    def set_fast_params(self, rows_per_batch: int = 0, filter_log2: int = 0, warps_per_block: int = 0) -> None:
        """Launch shape of the fast walk (0 = default): rows fetched per round trip, log2 of the
        recently-seen-id table's slots, warps per block.  Results do not depend on the shape."""
        _check(lib().pk_index_set_fast_params(self._h, rows_per_batch, filter_log2, warps_per_block))

    def set_fast_visited(self, log2_sets: int = 0) -> None:
        """The walk's second-level visited tables in L2: 0 = sized by list width (default),
        -1 = off, 1..20 = 2^log2_sets sets of eight tags per warp.  Results do not depend on it."""
        _check(lib().pk_index_set_fast_visited(self._h, int(log2_sets)))

    def set_build_walk(self, min_batch: int = 0) -> None:
        """Insertion batches of at least min_batch nodes take their layer-0 candidates from the FP16
        walk (0 = never, the default: the exact search for every batch)."""
        _check(lib().pk_index_set_build_walk(self._h, int(min_batch)))

    def set_fast_merge(self, min_winners: int = 0) -> None:
        """Wide lists merge a chunk's winners at once from min_winners of them (0 = by list width,
        -1 = never: one at a time).  Results do not depend on it."""
        _check(lib().pk_index_set_fast_merge(self._h, int(min_winners)))

    def set_fast_timing(self, enable: bool) -> None:
        """Record CUDA events around the walk and re-rank kernels of each fast search."""
        _check(lib().pk_index_set_fast_timing(self._h, int(bool(enable))))

    def fast_timing(self):
        """(walk_ms, rerank_ms) of the last timed fast search (waits for it)."""
        w = np.zeros(1, np.float32)
        r = np.zeros(1, np.float32)
        _check(lib().pk_index_fast_timing(self._h, _ptr(w), _ptr(r)))
        return float(w[0]), float(r[0])

    def tune_fast(self, queries, k: int, ef: int, expand: int = 1, stream=None):
        """Time a grid of walk launch shapes on this batch (a torch CUDA tensor), keep the fastest;
        returns ((rows_per_batch, filter_log2, warps_per_block), batch milliseconds)."""
        shape = np.zeros(3, np.int32)
        ms = np.zeros(1, np.float32)
        s = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _check(lib().pk_index_tune_fast(self._h, _dev_ptr(queries), queries.shape[0], k, ef, expand, _ptr(shape),
                                        _ptr(ms), s))
        return tuple(int(x) for x in shape), float(ms[0])

    def tune_fast_classes(self, queries, k: int, max_ef: int, expand: int = 1, stream=None):
        """Tune one walk launch shape per list-width class up to max_ef on these
        queries (a torch CUDA tensor), for batches with per-query ef; returns
        {class index: ((rows_per_batch, filter_log2, warps_per_block), ms)}."""
        shapes = np.zeros(30, np.int32)
        ms = np.zeros(10, np.float32)
        s = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _check(lib().pk_index_tune_fast_classes(self._h, _dev_ptr(queries), queries.shape[0], k, max_ef, expand,
                                                _ptr(shapes), _ptr(ms), s))
        return {c: (tuple(int(x) for x in shapes[3 * c:3 * c + 3]), float(ms[c])) for c in range(10)
                if shapes[3 * c] > 0}

    def set_fast_class_params(self, width_class: int, rows_per_batch: int = 0, filter_log2: int = 0,
                              warps_per_block: int = 0) -> None:
        """Launch shape of one list-width class (all zeros: the handle's shape)."""
        _check(lib().pk_index_set_fast_class_params(self._h, width_class, rows_per_batch, filter_log2,
                                                    warps_per_block))

    def search_fast_device(self, queries, k: int, ef: int, out_ids, out_dists, k_per_query=None, ef_per_query=None,
                           counters=None, expand: int = 1, stream=None) -> None:
        """Low-precision walk + exact re-rank on torch CUDA tensors (asynchronous)."""
        nq = queries.shape[0]
        s = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        _check(lib().pk_index_search_fast(self._h, _dev_ptr(queries), nq, k, ef, _dev_ptr(k_per_query),
                                          _dev_ptr(ef_per_query), out_ids.shape[1], _dev_ptr(out_ids),
                                          _dev_ptr(out_dists), _dev_ptr(counters), expand, s))

    def search_fast_var(self, queries: np.ndarray, k_per_query: np.ndarray, ef_per_query: np.ndarray,
                        expand: int = 1):
        """search_fast with a k and an ef per query: (ids, dists), nq x max(k)."""
        q = self._rows(queries)
        kq = np.ascontiguousarray(k_per_query, np.int32)
        eq = np.ascontiguousarray(ef_per_query, np.int32)
        if len(kq) != q.shape[0] or len(eq) != q.shape[0]:
            raise ValueError("one k and one ef per query")
        stride = int(kq.max()) if len(kq) else 1
        ids = np.empty((q.shape[0], stride), np.int32)
        dists = np.empty((q.shape[0], stride), np.float32)
        _check(lib().pk_index_search_fast_host_var(self._h, _ptr(q), q.shape[0], _ptr(kq), _ptr(eq), stride,
                                                   _ptr(ids), _ptr(dists), expand))
        return ids, dists

    def search_fast(self, queries: np.ndarray, k: int, ef: int, expand: int = 1):
        """Low-precision walk + exact re-rank with host buffers: (ids, dists)."""
        q = self._rows(queries)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.float32)
        _check(lib().pk_index_search_fast_host(self._h, _ptr(q), nq, k, ef, _ptr(ids), _ptr(dists), expand))
        return ids, dists

    # ---- persistence ----------------------------------------------------
    def save(self, path: str) -> None:
        _check(lib().pk_index_save(self._h, os.fsencode(path)))

    @_class_or_instance
    def load(cls, self, path: str) -> "HNSWIndex":
        """HNSWIndex.load(path) returns a new index read from a graph file;
        index.load(path) replaces this index's graph with the file's, as the
        reference binding's load does (pybind/hnsw.cpp:108-110)."""
        h = ctypes.c_void_p()
        _check(lib().pk_index_load(ctypes.byref(h), os.fsencode(path)))
        if self is None:
            return cls(_handle=h)
        self._deferred = False
        self._adopt(h)
        return self

    # ---- introspection --------------------------------------------------
    def info(self) -> dict:
        out = np.zeros(12, np.int64)
        _check(lib().pk_index_info(self._h, _ptr(out)))
        keys = ["n", "num_layers", "enter_level", "capacity", "dim", "M", "ef_construction", "metric", "dtype",
                "device_bytes", "cap0", "entry"]
        return {k: int(v) for k, v in zip(keys, out)}

    def layer(self, level: int) -> dict:
        n, lcap, cap = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().pk_index_layer(self._h, level, ctypes.byref(n), ctypes.byref(lcap), ctypes.byref(cap),
                                    None, None, None, None, None, None))
        n, lcap, cap = n.value, lcap.value, cap.value
        ext = np.empty(n, np.int32)
        deg = np.empty(n, np.int16)
        heu = np.empty(n, np.int16)
        hv = np.empty(n, np.uint8)
        adj = np.empty(lcap * cap, np.int32)
        dist = np.empty(lcap * cap, np.float32)
        _check(lib().pk_index_layer(self._h, level, ctypes.byref(ctypes.c_int64()), ctypes.byref(ctypes.c_int64()),
                                    ctypes.byref(ctypes.c_int64()), _ptr(ext), _ptr(deg), _ptr(heu), _ptr(hv),
                                    _ptr(adj), _ptr(dist)))
        return {"n": n, "layer_capacity": lcap, "cap": cap, "ext": ext, "degree": deg, "heuristic": heu,
                "has_vector": hv, "adj": adj, "dist": dist}

    def _rows(self, a: np.ndarray) -> np.ndarray:
        if self._h is None:
            raise RuntimeError("the index has not been built or loaded")
        a = np.ascontiguousarray(a)
        if a.ndim != 2 or a.shape[1] != self.dim:
            raise ValueError(f"expected (n, {self.dim}) rows, got {a.shape}")
        if a.dtype != self.dtype:
            raise TypeError(f"expected {self.dtype}, got {a.dtype}")
        return a


class Server:
    """Continuous-batching search server over an index (pk_server_* in the C ABI).

    Server(index, traversal="f16", slots=4, max_batch=4096, max_k=100, max_ef=256, device_bytes=0)
    submit(queries, k, ef) -> ticket (returns at once); wait(ticket) -> (ids, dists, latency_ms).
    Batches are admitted by device memory: device_bytes is the server's arena
    (0 = every slot's full batch at max_k and max_ef, at most half the free
    device memory); memory() reports its use and the requests that waited.
    """

    def __init__(self, index: "HNSWIndex", traversal: str = "f16", slots: int = 4, max_batch: int = 4096,
                 max_k: int = 100, max_ef: int = 256, expand: int = 1, device_bytes: int = 0):
        self.index = index
        self._s = None
        s = ctypes.c_void_p()
        _check(lib().pk_server_create_with_memory(ctypes.byref(s), index._h, HNSWIndex.TRAVERSAL[traversal], slots,
                                                  max_batch, max_k, max_ef, expand, device_bytes))
        self._s = s
        self._shape = {}

    def memory(self) -> dict:
        out = np.zeros(4, np.int64)
        _check(lib().pk_server_memory(self._s, _ptr(out)))
        return dict(zip(["arena_bytes", "in_use", "peak_in_use", "deferred_for_memory"], (int(x) for x in out)))

    def request_bytes(self, nq: int, k: int, ef: int) -> int:
        b = ctypes.c_int64()
        _check(lib().pk_server_request_bytes(self._s, nq, k, ef, ctypes.byref(b)))
        return b.value

    def submit(self, queries: np.ndarray, k: int, ef: int) -> int:
        q = self.index._rows(queries)
        t = ctypes.c_int64()
        _check(lib().pk_server_submit(self._s, _ptr(q), q.shape[0], k, ef, ctypes.byref(t)))
        self._shape[t.value] = (q.shape[0], k)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        nq, k = self._shape.pop(ticket)
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.float32)
        lat = ctypes.c_double()
        _check(lib().pk_server_wait(self._s, ticket, _ptr(ids), _ptr(dists), ctypes.byref(lat), timeout_ms))
        return ids, dists, lat.value

    def replay(self, queries: np.ndarray, nq: np.ndarray, arrival_us: np.ndarray, k: np.ndarray, ef: np.ndarray,
               out_stride: int = 0):
        """Replay a timed trace natively; returns (ids, dists, latency_ms per request)."""
        q = self.index._rows(queries)
        nq = np.ascontiguousarray(nq, np.int32)
        arr = np.ascontiguousarray(arrival_us, np.float64)
        k = np.ascontiguousarray(k, np.int32)
        ef = np.ascontiguousarray(ef, np.int32)
        n = len(nq)
        stride = out_stride or int(k.max())
        ids = np.full((int(nq.sum()), stride), -1, np.int32)
        dists = np.full((int(nq.sum()), stride), np.inf, np.float32)
        lat = np.zeros(n, np.float64)
        _check(lib().pk_server_replay(self._s, _ptr(q), n, _ptr(nq), _ptr(arr), _ptr(k), _ptr(ef), _ptr(ids),
                                      _ptr(dists), stride, _ptr(lat)))
        return ids, dists, lat

    def set_watchdog(self, seconds: float) -> None:
        _check(lib().pk_server_set_watchdog(self._s, seconds))

    def stats(self) -> dict:
        out = np.zeros(5, np.int64)
        _check(lib().pk_server_stats(self._s, _ptr(out)))
        return dict(zip(["batches", "queries", "max_inflight", "queued", "error"], (int(x) for x in out)))

    def close(self) -> None:
        if getattr(self, "_s", None):
            lib().pk_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the module's globals may be gone
            pass
