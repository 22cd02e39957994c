"""Device insertion (batched build) against the oracle and the reference.

With one node per batch the device build is the reference's one-thread build
with adjacency lists bounded by their caps, which the oracle restates as
GROWTH_CAPPED: on integer data the two graphs must be identical array by
array.  With large batches the graph differs (nodes of a batch do not see each
other), and the bar is recall: searching it must reach the recall of a graph
built by the reference's own code at the same M, ef_construction and ef.
"""
import numpy as np
import pytest

import oracle
from pickle_b200 import HNSWIndex, datasets
from tests.helpers import build_recall_tolerance, case_data, levels_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["f32int_l2", "u8_ip", "i8_l2_d100", "f32unit_ip", "f16_l2"])
def test_one_node_batches_equal_oracle_build(name, gpu):
    """Float data too: the restatement builds with the device's float
    summation order (the only difference between the two), and then every
    array and every search answer is identical."""
    metric, base, queries, M, efc = case_data(name)
    n = 1500
    base = base[:n]
    order = np.random.default_rng(5).permutation(n).astype(np.int32)
    lv = levels_for(n, M, 5)
    g = oracle.OraGraph.new(metric, base.dtype, base.shape[1], M, efc, lv, oracle.GROWTH_CAPPED)
    with oracle.float_order(oracle.ORDER_DEVICE):
        g.build(base, order)
    idx = HNSWIndex(base.shape[1], base.dtype, metric, M, efc)
    idx.set_levels(lv)
    idx.build(base, order, max_batch=1)
    info = idx.info()
    oinfo = g.info()
    assert info["n"] == oinfo["n0"] and info["num_layers"] == oinfo["num_layers"]
    assert info["enter_level"] == oinfo["enter_level"]
    for level in range(oinfo["num_layers"]):
        a, b = idx.layer(level), g.layer(level)
        n_l, cap = b["n"], b["cap"]
        assert a["n"] == n_l and a["cap"] == cap
        np.testing.assert_array_equal(a["ext"], b["ext"])
        np.testing.assert_array_equal(a["degree"], b["degree"])
        np.testing.assert_array_equal(a["heuristic"], b["heuristic"])
        np.testing.assert_array_equal(a["adj"][:n_l * cap], b["adj"][:n_l * cap])
        np.testing.assert_array_equal(a["dist"][:n_l * cap], b["dist"][:n_l * cap])
    # and the two graphs answer queries identically
    with oracle.float_order(oracle.ORDER_DEVICE):
        oi, od = g.search(queries, 10, 40)
    ids, ds = idx.search(queries, 10, 40)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(ds, od)


def test_saved_build_reloads_identically(gpu, tmp_path):
    metric, base, queries, M, efc = case_data("u8_l2")
    idx = HNSWIndex(base.shape[1], base.dtype, metric, M, efc)
    idx.set_seed(11)
    idx.build(base)
    p = str(tmp_path / "g.pkg")
    idx.save(p)
    ids, ds = idx.search(queries, 10, 40)
    again = HNSWIndex.load(p)
    i2, d2 = again.search(queries, 10, 40)
    np.testing.assert_array_equal(ids, i2)
    np.testing.assert_array_equal(ds, d2)
    # the device library writes version 2 (block checksum) and checks it on load
    raw = open(p, "rb").read()
    assert int.from_bytes(raw[8:12], "little") == 2
    from tests.test_oracle_pins import v2_checksum
    assert int.from_bytes(raw[-8:], "little") == v2_checksum(raw[:-8])
    bad = bytearray(raw)
    bad[len(bad) // 2] ^= 4
    open(p + ".bad", "wb").write(bytes(bad))
    with pytest.raises(Exception):
        HNSWIndex.load(p + ".bad")
    # the oracle reads the device library's file and answers the same
    g = oracle.OraGraph.load(p)
    oi, od = g.search(queries, 10, 40)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(ds, od)


@pytest.mark.parametrize("name", ["f32int_l2", "f32unit_ip"])
def test_batched_build_reaches_reference_recall(name, gpu, ref_bin, tmp_path):
    """Three batched device builds (seeds 3-5) against three builds by the
    reference's parallel Build (level draws from seeds 0-2): the device graphs'
    mean recall@10 is at least the reference graphs' mean minus two standard
    errors of the difference (the graphs' spread over seeds and the sampling
    error of a recall over 200 queries x 10)."""
    metric, base, queries, M, efc = case_data(name)
    n = len(base)
    gt, _ = datasets.exact_knn(base, queries, 10, metric)
    efs = (16, 32, 64)
    r_ref = {ef: [] for ef in efs}
    r_dev = {ef: [] for ef in efs}
    for s in range(3):
        rpath = str(tmp_path / f"ref{s}.pkg")
        oracle.ref_build(base, metric, M, efc, rpath, threads=8, levels=levels_for(n, M, s))
        idx = HNSWIndex(base.shape[1], base.dtype, metric, M, efc)
        idx.set_seed(3 + s)
        idx.build(base)
        for ef in efs:
            ri, _, _ = oracle.ref_search(rpath, queries, 10, ef, threads=4)
            ids, _ = idx.search(queries, 10, ef)
            r_ref[ef].append(datasets.recall_at_k(ri, gt, 10))
            r_dev[ef].append(datasets.recall_at_k(ids, gt, 10))
        idx.close()
    for ef in efs:
        tol = build_recall_tolerance(r_ref[ef], r_dev[ef], 10 * len(queries))
        assert np.mean(r_dev[ef]) >= np.mean(r_ref[ef]) - tol, (ef, r_dev[ef], r_ref[ef], tol)


@pytest.mark.parametrize("min_batch", [256, 1])
def test_walk_assisted_build_keeps_recall(min_batch, gpu):
    """Insertion batches that take their layer-0 candidates from the FP16 walk
    (batches of 256 nodes or more, or every batch with min_batch = 1) build a
    graph nearly as good as the exact-search build of the same rows and
    levels: recall@10 at equal ef within 0.01."""
    base, queries = datasets.gmm_f16(20000, 300, 64, ncomp=32, sigma=0.5, seed=21)
    gt, _ = datasets.exact_knn(base, queries, 10, "l2")
    rec = {}
    for mode in (min_batch, 0):
        idx = HNSWIndex(64, np.float16, "l2", M=16, ef_construction=100)
        idx.set_seed(21)
        idx.set_build_walk(mode)
        idx.build(base)
        rec[mode] = {ef: datasets.recall_at_k(idx.search(queries, 10, ef)[0], gt, 10) for ef in (16, 32, 64)}
        idx.close()
    for ef in (16, 32, 64):
        assert rec[min_batch][ef] >= rec[0][ef] - 0.01, (ef, rec)
    assert rec[min_batch][64] >= 0.95, rec
