"""Seeded synthetic datasets with the shapes and value distributions of the
benchmark configurations (the public datasets the reference benchmarks on,
benchmark/bench_util.hpp:250-263, are not available offline).

Every generator returns (base, queries) as numpy arrays and is a pure function
of its arguments.
"""
from __future__ import annotations

import numpy as np


def gmm_int_f32(n: int, nq: int, dim: int = 128, ncomp: int = 64, sigma: float = 20.0, seed: int = 0):
    """Integer-valued float32 in [0, 255] from a Gaussian mixture: component
    centres uniform in [0, 255], per-coordinate sigma, rounded and clipped.
    Squared L2 distances between such rows are exact integers below 2^24 for
    dim <= 258, so float32 results do not depend on summation order."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 255, size=(ncomp, dim))
    lab = rng.integers(0, ncomp, size=n + nq)
    x = np.clip(np.rint(centres[lab] + rng.normal(0, sigma, size=(n + nq, dim))), 0, 255).astype(np.float32)
    return x[:n], x[n:]


def gmm_unit(n: int, nq: int, dim: int = 96, ncomp: int = 256, sigma: float = 0.3, seed: int = 0,
             dtype=np.float32, zipf_s: float | None = None):
    """Unit-normalised rows from a Gaussian mixture around random unit centres
    (for inner product).  With zipf_s the cluster sizes are Zipf-distributed."""
    rng = np.random.default_rng(seed)
    centres = rng.normal(size=(ncomp, dim))
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    if zipf_s is None:
        lab = rng.integers(0, ncomp, size=n + nq)
    else:
        w = 1.0 / np.arange(1, ncomp + 1) ** zipf_s
        lab = rng.choice(ncomp, size=n + nq, p=w / w.sum())
    # filled chunk by chunk in the target type (rounded through float32 as a
    # whole-array conversion would be), so large float16 sets never hold a
    # float32 copy
    x = np.empty((n + nq, dim), dtype)
    step = 1 << 18
    for i in range(0, n + nq, step):
        j = min(n + nq, i + step)
        y = centres[lab[i:j]] + rng.normal(0, sigma / np.sqrt(dim), size=(j - i, dim))
        y /= np.linalg.norm(y, axis=1, keepdims=True)
        x[i:j] = y.astype(np.float32).astype(dtype)
    return x[:n], x[n:]


def embedding_like(n: int, nq: int, dim: int = 768, ncomp: int = 2048, zipf_s: float = 1.1, rank: int = 48,
                   spread: float = 0.6, seed: int = 0, dtype=np.float16):
    """Unit rows shaped like text embeddings: mixture components with
    Zipf(zipf_s)-distributed sizes around random unit centres, each spread
    over its own random rank-`rank` subspace with a decaying spectrum
    (standard deviations proportional to 1/sqrt(i+1), total norm `spread`),
    then normalised.  Embedding sets have a low intrinsic dimension; an
    isotropic 768-dimensional spread instead makes every point nearly
    equidistant from its cluster-mates, which no graph index searches well."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((ncomp, dim)).astype(np.float32)
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    w = 1.0 / np.arange(1, ncomp + 1) ** zipf_s
    lab = rng.choice(ncomp, size=n + nq, p=w / w.sum())
    sv = 1.0 / np.sqrt(np.arange(1, rank + 1))
    sv = (spread * sv / np.linalg.norm(sv)).astype(np.float32)
    x = np.empty((n + nq, dim), dtype)
    order = np.argsort(lab, kind="stable")
    bounds = np.searchsorted(lab[order], np.arange(ncomp + 1))
    for c in range(ncomp):
        rows = order[bounds[c]:bounds[c + 1]]
        if len(rows) == 0:
            continue
        basis, _ = np.linalg.qr(rng.standard_normal((dim, rank)).astype(np.float32))
        for i in range(0, len(rows), 1 << 16):
            r = rows[i:i + (1 << 16)]
            z = rng.standard_normal((len(r), rank)).astype(np.float32) * sv
            y = centres[c] + z @ basis.T
            y /= np.linalg.norm(y, axis=1, keepdims=True)
            x[r] = y.astype(dtype)
    return x[:n], x[n:]


def gmm_bytes(n: int, nq: int, dim: int = 128, ncomp: int = 64, sigma: float = 12.0, signed: bool = False,
              seed: int = 0):
    """uint8 or int8 rows: mixture centres uniform over the type's range,
    per-coordinate Gaussian noise, rounded and clipped to the range."""
    rng = np.random.default_rng(seed)
    lo, hi = (-128, 127) if signed else (0, 255)
    centres = rng.uniform(lo, hi, size=(ncomp, dim))
    lab = rng.integers(0, ncomp, size=n + nq)
    x = np.clip(np.rint(centres[lab] + rng.normal(0, sigma, size=(n + nq, dim))), lo, hi)
    x = x.astype(np.int8 if signed else np.uint8)
    return x[:n], x[n:]


def gmm_f16(n: int, nq: int, dim: int = 128, ncomp: int = 1024, sigma: float = 0.5, seed: int = 0):
    """float16 rows from a Gaussian mixture with unit-normal centres."""
    rng = np.random.default_rng(seed)
    centres = rng.normal(size=(ncomp, dim)).astype(np.float32)
    lab = rng.integers(0, ncomp, size=n + nq)
    x = np.empty((n + nq, dim), np.float16)
    step = 1 << 18
    for i in range(0, n + nq, step):
        j = min(n + nq, i + step)
        x[i:j] = (centres[lab[i:j]] + rng.normal(0, sigma, size=(j - i, dim)).astype(np.float32)).astype(np.float16)
    return x[:n], x[n:]


def exact_knn(base: np.ndarray, queries: np.ndarray, k: int, metric: str = "l2"):
    """Exact k nearest neighbours in float64 (small inputs; numpy).  Ties are
    broken by id.  Returns (ids, dists) with the index's distance convention
    (squared L2, or negative inner product)."""
    b = base.astype(np.float64)
    q = queries.astype(np.float64)
    ids = np.empty((len(q), k), np.int64)
    ds = np.empty((len(q), k), np.float64)
    bn = (b * b).sum(1)
    for i in range(0, len(q), 256):
        qq = q[i:i + 256]
        if metric == "l2":
            d = (qq * qq).sum(1)[:, None] + bn[None, :] - 2 * qq @ b.T
        else:
            d = -(qq @ b.T)
        part = np.argpartition(d, min(k, d.shape[1] - 1), axis=1)[:, :k]
        for r in range(len(qq)):
            cand = part[r]
            order = np.lexsort((cand, d[r, cand]))
            ids[i + r] = cand[order]
            ds[i + r] = d[r, cand[order]]
    return ids, ds


def recall_at_k(found: np.ndarray, truth: np.ndarray, k: int) -> float:
    """Label-match recall@k as the reference's benchmark computes it
    (benchmark/hnsw_pickle.cpp:94-112)."""
    hit = 0
    for f, t in zip(found[:, :k], truth[:, :k]):
        hit += len(set(int(x) for x in f if x >= 0) & set(int(x) for x in t))
    return hit / (k * len(found))
