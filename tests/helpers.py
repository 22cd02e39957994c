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


def mismatched_queries(ids_a, d_a, ids_b, d_b, rel=1e-6):
    """Indices of the queries whose id lists differ somewhere other than at a
    tie (two distances within rel of each other at that position)."""
    out = []
    for qi, (ia, da, ib, db) in enumerate(zip(ids_a, d_a, ids_b, d_b)):
        for x, dx, y, dy in zip(ia, da, ib, db):
            if x != y and abs(float(dx) - float(dy)) > rel * max(abs(float(dx)), abs(float(dy)), 1e-30):
                out.append(qi)
                break
    return out


def reference_distance_table(base, queries, touched, metric):
    """The reference binary's own distances (pk_ref dist, the instantiation its
    search runs) from each query to the rows its search touched; keys are
    external ids, -1 the zero row.  Returns the (offsets, keys, values) table
    of OraGraph.search_fork."""
    keys = [np.unique(t) for t in touched]
    off = np.zeros(len(keys) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in keys])
    K = np.concatenate(keys).astype(np.int32) if keys else np.zeros(0, np.int32)
    qi = np.repeat(np.arange(len(keys)), [len(x) for x in keys])
    rows = base[np.maximum(K, 0)].copy()
    rows[K < 0] = 0
    vals = oracle.ref_dist(metric, np.ascontiguousarray(queries[qi]), rows)
    return off, K, vals.astype(np.float32)


def float_parity(graph_path, base, queries, metric, k, ef, ids, dists, other_ids, other_dists, other="source",
                 rel=1e-6, touched_cap=200_000):
    """Float parity of device results (ids, dists) on a saved graph.

    1. The restatement replayed with the device's float summation order must
       return exactly the device's ids and distances (asserted here): the
       device runs the reference's algorithm and differs only in rounding.
    2. Against `other` (the restatement in the reference's source order, or
       the reference binary itself: other = "reference"), the queries whose
       ids differ beyond ties within rel are counted, and each is replayed
       by the fork detector with the device's distances driving and the
       other side's distances compared: the first decision that flips is the
       fork, and its two operands' relative gap is returned.
    Returns {"queries", "mismatched", "gaps": [(where, gap_device, gap_other)]}."""
    g = oracle.OraGraph.load(graph_path)
    with oracle.float_order(oracle.ORDER_DEVICE):
        oi, od = g.search(queries, k, ef, threads=8)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(dists, od)
    bad = mismatched_queries(ids, dists, other_ids, other_dists, rel)
    gaps = []
    if bad:
        qs = np.ascontiguousarray(queries[bad])
        if other == "source":
            _, _, fork, _ = g.search_fork(qs, k, ef, oracle.ORDER_DEVICE, oracle.ORDER_SOURCE, threads=8)
        else:
            _, _, _, touched = g.search_fork(qs, k, ef, oracle.ORDER_DEVICE, oracle.ORDER_DEVICE, threads=8,
                                             touched_cap=touched_cap)
            table = reference_distance_table(base, qs, touched, metric)
            _, _, fork, _ = g.search_fork(qs, k, ef, oracle.ORDER_DEVICE, oracle.ORDER_TABLE, table=table, threads=8)
        for f in fork:
            assert f[0] == 1.0 and f[1] != 5, f"a mismatched query did not fork inside the search: {f}"
            ga = abs(f[2] - f[3]) / max(abs(f[2]), abs(f[3]), 1e-30)
            gb = abs(f[4] - f[5]) / max(abs(f[4]), abs(f[5]), 1e-30)
            gaps.append((int(f[1]), ga, gb))
    return {"queries": len(ids), "mismatched": len(bad), "gaps": gaps}


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


def build_recall_tolerance(ref_recalls, dev_recalls, labels):
    """Two standard errors of (mean device-graph recall - mean reference-graph
    recall), each side's mean taken over graphs built from different seeds:
    the graphs' spread around their mean (sample variance over seeds, when
    there are several) plus the sampling error of one recall over `labels`
    binary outcomes (queries x k)."""
    r = np.asarray(ref_recalls, np.float64)
    d = np.asarray(dev_recalls, np.float64)
    m = float(r.mean())
    samp = max(m * (1.0 - m), 1e-4) / labels
    var = samp / len(r) + samp / len(d)
    if len(r) > 1:
        var += r.var(ddof=1) / len(r)
    if len(d) > 1:
        var += d.var(ddof=1) / len(d)
    return 2.0 * float(np.sqrt(var))
