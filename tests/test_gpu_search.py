"""Parity of the device search (plain, exact path) with the oracle and the
reference's own search, on graphs built by the reference's own code.

Bar: integer data (and integer-valued float32, whose L2 distances are exact
in any summation order) must match bit for bit in ids, distances and the
per-level work counters.  Float data must give identical ids except for ties
within 1e-6 relative distance, and the same recall@k within 0.001.
"""
import numpy as np
import pytest

import oracle
from pickle_b200 import HNSWIndex, datasets
from tests.helpers import CASES, INTEGER_CASES, case_data, float_parity, ref_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("ef", [10, 33, 48])
def test_search_matches_oracle(name, ef, gpu, ref_bin):
    """Integer cases: bit for bit.  Float cases: the restatement replayed with
    the device's summation order returns exactly the device's ids and
    distances; against the restatement in the reference's source order, every
    query whose ids differ beyond ties within 1e-6 forks at a comparison of two
    distances within 1e-6 of each other, and recall@k is equal within 0.001."""
    metric, base, queries, M, efc = case_data(name)
    path = ref_graph(name)
    g = oracle.OraGraph.load(path)
    k = 10
    oi, od, ocnt = g.search(queries, k, ef, threads=4, counters=True)
    idx = HNSWIndex.load(path)
    ids, dists = idx.search(queries, k, ef)
    if name in INTEGER_CASES:
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(dists, od)
    else:
        rep = float_parity(path, base, queries, metric, k, ef, ids, dists, oi, od, other="source")
        for where, gap_dev, gap_src in rep["gaps"]:
            assert min(gap_dev, gap_src) <= 1e-6, (where, gap_dev, gap_src)
        gt, _ = datasets.exact_knn(base, queries, k, metric)
        r_dev = datasets.recall_at_k(ids, gt, k)
        r_ora = datasets.recall_at_k(oi, gt, k)
        assert abs(r_dev - r_ora) <= 0.001 + 1.0 / (k * len(queries)), (r_dev, r_ora)


@pytest.mark.parametrize("name", sorted(set(CASES) - INTEGER_CASES))
def test_float_search_vs_reference_binary(name, gpu, ref_bin):
    """Float data against the reference's own AnnSearch on the same file: the
    queries whose ids differ beyond 1e-6 ties are counted, each is shown to
    fork at a near-tie of the two sides' own distances (the reference's are
    taken from its binary), and recall@10 agrees within 0.001."""
    metric, base, queries, M, efc = case_data(name)
    path = ref_graph(name)
    ri, rd, _ = oracle.ref_search(path, queries, 10, 32, threads=4)
    idx = HNSWIndex.load(path)
    ids, dists = idx.search(queries, 10, 32)
    rep = float_parity(path, base, queries, metric, 10, 32, ids, dists, ri, rd, other="reference")
    assert rep["mismatched"] <= 0.05 * len(queries), rep
    for where, gap_dev, gap_ref in rep["gaps"]:
        assert min(gap_dev, gap_ref) <= 1e-6, (where, gap_dev, gap_ref)
    gt, _ = datasets.exact_knn(base, queries, 10, metric)
    assert abs(datasets.recall_at_k(ids, gt, 10) - datasets.recall_at_k(ri, gt, 10)) <= 0.001 + 1.0 / (
        10 * len(queries))


@pytest.mark.parametrize("name", sorted(INTEGER_CASES))
def test_search_matches_reference_binary(name, gpu, ref_bin):
    """Against the reference's own AnnSearch run on the same file."""
    metric, base, queries, M, efc = case_data(name)
    path = ref_graph(name)
    ri, rd, info = oracle.ref_search(path, queries, 10, 32, threads=4, metrics=True)
    idx = HNSWIndex.load(path)
    ids, dists = idx.search(queries, 10, 32)
    np.testing.assert_array_equal(ids, ri)
    np.testing.assert_array_equal(dists, rd)


@pytest.mark.parametrize("name", ["f32int_l2", "u8_ip", "i8_l2_d100"])
def test_counters_match_oracle(name, gpu, ref_bin):
    import torch
    metric, base, queries, M, efc = case_data(name)
    path = ref_graph(name)
    g = oracle.OraGraph.load(path)
    oi, od, ocnt = g.search(queries, 10, 40, threads=4, counters=True)
    idx = HNSWIndex.load(path)
    q = torch.from_numpy(queries).cuda()
    ids = torch.empty((len(queries), 10), dtype=torch.int32, device="cuda")
    ds = torch.empty((len(queries), 10), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((len(queries), 6), dtype=torch.int32, device="cuda")
    idx.search_device(q, 10, 40, ids, ds, counters=cnt)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ids.cpu().numpy(), oi)
    np.testing.assert_array_equal(cnt.cpu().numpy(), ocnt.astype(np.int32))


def test_mixed_k_ef_batch_equals_uniform(gpu, ref_bin):
    """Per-query k and ef in one launch give the same rows as uniform launches."""
    import torch
    metric, base, queries, M, efc = case_data("u8_l2")
    idx = HNSWIndex.load(ref_graph("u8_l2"))
    rng = np.random.default_rng(3)
    nq = len(queries)
    ks = rng.choice([1, 5, 10, 20], size=nq).astype(np.int32)
    efs = rng.integers(20, 90, size=nq).astype(np.int32)
    stride = int(ks.max())
    q = torch.from_numpy(queries).cuda()
    ids = torch.full((nq, stride), -7, dtype=torch.int32, device="cuda")
    ds = torch.zeros((nq, stride), dtype=torch.float32, device="cuda")
    idx.search_device(q, stride, int(efs.max()), ids, ds, k_per_query=torch.from_numpy(ks).cuda(),
                      ef_per_query=torch.from_numpy(efs).cuda())
    torch.cuda.synchronize()
    ids, ds = ids.cpu().numpy(), ds.cpu().numpy()
    for i in range(0, nq, 7):
        ui, ud = idx.search(queries[i:i + 1], int(ks[i]), int(efs[i]))
        np.testing.assert_array_equal(ids[i, :ks[i]], ui[0])
        np.testing.assert_array_equal(ds[i, :ks[i]], ud[0])


def test_k_larger_than_results_pads(gpu, ref_bin):
    metric, base, queries, M, efc = case_data("i8_ip")
    path = ref_graph("i8_ip")
    g = oracle.OraGraph.load(path)
    oi, od = g.search(queries[:20], 60, 30)
    ids, dists = HNSWIndex.load(path).search(queries[:20], 60, 30)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(dists, od)
    assert (ids[:, 30:] == -1).all()
