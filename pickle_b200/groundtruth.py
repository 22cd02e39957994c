"""Exact k nearest neighbours on the GPU for benchmark-sized inputs.

The base is held on the device in its own type.  Candidates come from
float32 matrix products (TF32 off) over chunks of the queries and of the
base: the best k + 32 by float32 score across all chunks are re-scored in
float64 and ordered by (distance, id).  The distance convention is the
index's: squared L2, or negative inner product.  Used by the benchmark
drivers, not by the search path.
"""
from __future__ import annotations

import numpy as np


def gpu_knn(base: np.ndarray, queries: np.ndarray, k: int, metric: str, device=None, qchunk: int = 1024,
            bchunk: int = 1 << 20) -> np.ndarray:
    """Ids (int64, nq x k) of the exact k nearest rows of base."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    dev = device or torch.device("cuda")
    bg = torch.from_numpy(np.ascontiguousarray(base)).to(dev)
    nb = bg.shape[0]
    norms = None
    if metric == "l2":
        norms = torch.cat([(bg[i:i + bchunk].float() ** 2).sum(1) for i in range(0, nb, bchunk)])
    keep = min(k + 32, nb)
    out = np.empty((len(queries), k), np.int64)
    for q0 in range(0, len(queries), qchunk):
        q = torch.from_numpy(np.ascontiguousarray(queries[q0:q0 + qchunk])).to(dev).float()
        vals, idxs = [], []
        for i in range(0, nb, bchunk):
            b = bg[i:i + bchunk].float()
            s = -(q @ b.T) if metric == "ip" else (q * q).sum(1)[:, None] + norms[None, i:i + bchunk] - 2.0 * (q @ b.T)
            v, ix = torch.topk(s, min(keep, b.shape[0]), dim=1, largest=False)
            vals.append(v)
            idxs.append(ix + i)
        v = torch.cat(vals, dim=1)
        ix = torch.cat(idxs, dim=1)
        sel = torch.topk(v, keep, dim=1, largest=False).indices
        cand = torch.gather(ix, 1, sel)
        rows = bg[cand].double()
        qd = q.double()[:, None, :]
        d = -(qd * rows).sum(-1) if metric == "ip" else ((qd - rows) ** 2).sum(-1)
        order = torch.argsort(cand, dim=1, stable=True)
        d, cand = torch.gather(d, 1, order), torch.gather(cand, 1, order)
        order = torch.argsort(d, dim=1, stable=True)[:, :k]
        out[q0:q0 + len(q)] = torch.gather(cand, 1, order).cpu().numpy()
    return out
