"""Shared test helpers: seeded datasets, reference-built graphs, comparisons."""
from __future__ import annotations

import functools
import os
import tempfile

import numpy as np

import oracle
from pickle_b200 import datasets

_TMP = tempfile.mkdtemp(prefix="pk_tests_")

# name -> (metric, generator, n, nq, dim, M, efc)
CASES = {
    "f32int_l2": ("l2", lambda n, q, d, s: datasets.gmm_int_f32(n, q, d, ncomp=16, seed=s), 4000, 200, 32, 8, 64),
    "f32unit_ip": ("ip", lambda n, q, d, s: datasets.gmm_unit(n, q, d, ncomp=32, seed=s), 4000, 200, 48, 8, 64),
    "f32_l2_d96": ("l2", lambda n, q, d, s: datasets.gmm_unit(n, q, d, ncomp=32, seed=s), 3000, 200, 96, 12, 80),
    "u8_l2": ("l2", lambda n, q, d, s: datasets.gmm_bytes(n, q, d, ncomp=16, seed=s), 4000, 200, 64, 8, 64),
    "u8_ip": ("ip", lambda n, q, d, s: datasets.gmm_bytes(n, q, d, ncomp=16, seed=s), 3000, 200, 64, 8, 48),
    "i8_l2_d100": ("l2", lambda n, q, d, s: datasets.gmm_bytes(n, q, d, ncomp=16, signed=True, seed=s), 4000, 200,
                   100, 8, 64),
    "i8_ip": ("ip", lambda n, q, d, s: datasets.gmm_bytes(n, q, d, ncomp=16, signed=True, seed=s), 3000, 200, 32, 6,
              40),
    "f16_l2": ("l2", lambda n, q, d, s: datasets.gmm_f16(n, q, d, ncomp=32, seed=s), 3000, 200, 64, 8, 64),
    "f16_ip_d768": ("ip", lambda n, q, d, s: datasets.gmm_unit(n, q, d, ncomp=16, seed=s, dtype=np.float16), 1500,
                    100, 768, 8, 48),
}
INTEGER_CASES = {"f32int_l2", "u8_l2", "u8_ip", "i8_l2_d100", "i8_ip"}


def levels_for(n: int, M: int, seed: int) -> np.ndarray:
    """Levels with the reference's distribution (include/util.hpp:13-64)."""
    cp = oracle.cumulative_probability(M)
    rng = np.random.default_rng(seed + 12345)
    u = rng.random((n, len(cp)))
    hit = u < cp[None, :]
    lv = np.where(hit.any(1), hit.argmax(1), len(cp) - 1)
    return lv.astype(np.uint8)


@functools.lru_cache(maxsize=None)
def case_data(name: str, seed: int = 0):
    metric, gen, n, nq, dim, M, efc = CASES[name]
    base, queries = gen(n, nq, dim, seed)
    return metric, base, queries, M, efc


@functools.lru_cache(maxsize=None)
def ref_graph(name: str, seed: int = 0, threads: int = 1) -> str:
    """A graph built by the reference's own code (one thread, fixed levels
    and order), saved as a v2 file."""
    metric, base, queries, M, efc = case_data(name, seed)
    n = len(base)
    order = np.random.default_rng(seed + 7).permutation(n).astype(np.int32)
    path = os.path.join(_TMP, f"{name}_{seed}_{threads}.pkg")
    oracle.ref_build(base, metric, M, efc, path, threads=threads, order=order, levels=levels_for(n, M, seed))
    return path


def compare_float_results(ids_a, d_a, ids_b, d_b, rel=1e-6):
    """Fraction of queries whose id lists agree, where a mismatch counts as
    agreement when the two distances at that position are within rel of each
    other (a tie)."""
    ok = 0
    for ia, da, ib, db in zip(ids_a, d_a, ids_b, d_b):
        same = True
        for x, dx, y, dy in zip(ia, da, ib, db):
            if x != y and abs(float(dx) - float(dy)) > rel * max(abs(float(dx)), abs(float(dy)), 1e-30):
                same = False
                break
        ok += same
    return ok / len(ids_a)
