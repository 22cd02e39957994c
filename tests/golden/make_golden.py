"""Regenerate the golden fixtures from the reference's own code.

    python tests/golden/make_golden.py        (needs oracle/_ref/pk_ref)

For each case it stores, produced by oracle/_ref/pk_ref (the reference's
headers compiled unmodified):
  <case>.pkg  the graph of a one-thread reference Build with the given levels
              and insertion order (its exact output);
  <case>.npz  data, order, levels, queries, and the reference's AnnSearch
              ids / distances at k=10, ef=32 on that graph, plus its
              per-level work counters.
The cases are small (600 nodes) so the fixtures stay a few hundred KB.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from pickle_b200 import datasets  # noqa: E402

CASES = {
    "f32int_l2": ("l2", lambda: datasets.gmm_int_f32(600, 50, 24, ncomp=8, seed=21), 6, 40),
    "u8_ip": ("ip", lambda: datasets.gmm_bytes(600, 50, 32, ncomp=8, seed=22), 6, 40),
    "i8_l2_d100": ("l2", lambda: datasets.gmm_bytes(600, 50, 100, ncomp=8, signed=True, seed=23), 6, 40),
    "f16_ip": ("ip", lambda: datasets.gmm_unit(600, 50, 32, ncomp=8, seed=24, dtype=np.float16), 6, 40),
}


def levels_for(n, M, seed):
    cp = oracle.cumulative_probability(M)
    rng = np.random.default_rng(seed)
    u = rng.random((n, len(cp)))
    hit = u < cp[None, :]
    return np.where(hit.any(1), hit.argmax(1), len(cp) - 1).astype(np.uint8)


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/pk_ref is not built (make -f oracle/Makefile)")
    for name, (metric, gen, M, efc) in CASES.items():
        data, queries = gen()
        n = len(data)
        order = np.random.default_rng(100).permutation(n).astype(np.int32)
        levels = levels_for(n, M, 200)
        gpath = os.path.join(HERE, name + ".pkg")
        oracle.ref_build(data, metric, M, efc, gpath, threads=1, order=order, levels=levels)
        ids, dists, info = oracle.ref_search(gpath, queries, 10, 32, threads=1, metrics=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), data=data, order=order, levels=levels,
                            queries=queries, ids=ids, dists=dists,
                            meta=np.array(json.dumps({"metric": metric, "M": M, "efc": efc, "k": 10, "ef": 32,
                                                      "counters": info})))
        print(name, os.path.getsize(gpath), "bytes")


if __name__ == "__main__":
    main()
