"""Parity at the size of the first benchmark configuration.

100k x 128 integer-valued float32 rows (64-component mixture, centres in
[0, 255], sigma 20, rounded and clipped), L2, M = 16, ef_construction = 200,
graph built by the reference's own parallel Build (include/hnsw.hpp:497-507)
on the host, 10k queries from the same mixture, k = 10.  Squared L2 between
such rows is an integer below 2^24, exact in any summation order, so at every
ef of the configuration's sweep the device search must equal the reference
binary's batch AnnSearch (include/hnsw.hpp:528-541) bit for bit: ids,
distances, and the per-level work counters of its collect_metric pass
(include/profiler.hpp:60-68).
"""
import numpy as np
import pytest

import oracle
from pickle_b200 import HNSWIndex, datasets

pytestmark = pytest.mark.gpu

N, NQ, DIM, M, EFC, K = 100_000, 10_000, 128, 16, 200, 10


@pytest.fixture(scope="module")
def c1(tmp_path_factory, ref_bin):
    base, queries = datasets.gmm_int_f32(N, NQ, DIM, ncomp=64, sigma=20.0, seed=0)
    path = str(tmp_path_factory.mktemp("c1") / "c1_ref.pkg")
    oracle.ref_build(base, "l2", M, EFC, path)
    return base, queries, path


@pytest.mark.parametrize("ef", [16, 32, 64, 128, 256])
def test_c1_search_equals_reference_binary(c1, ef, gpu):
    import torch
    base, queries, path = c1
    ri, rd, info = oracle.ref_search(path, queries, K, ef, metrics=True)
    idx = HNSWIndex.load(path)
    q = torch.from_numpy(queries).cuda()
    ids = torch.empty((NQ, K), dtype=torch.int32, device="cuda")
    ds = torch.empty((NQ, K), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((NQ, 6), dtype=torch.int32, device="cuda")
    idx.search_device(q, K, ef, ids, ds, counters=cnt)
    torch.cuda.synchronize()
    ids, ds, cnt = ids.cpu().numpy(), ds.cpu().numpy(), cnt.cpu().numpy().astype(np.int64)
    np.testing.assert_array_equal(ids, ri)
    np.testing.assert_array_equal(ds, rd)
    assert cnt[:, 0].sum() + cnt[:, 3].sum() == info["hop"]
    assert cnt[:, 1].sum() + cnt[:, 4].sum() == info["dist"]
    assert cnt[:, 3].sum() == info["base_hop"]
    assert cnt[:, 4].sum() == info["base_dist"]
    assert cnt[:, 2].sum() + cnt[:, 5].sum() == info["neighbor"]
    # the host entry point (pk_index_search) returns the same
    hi, hd = idx.search(queries[:2000], K, ef)
    np.testing.assert_array_equal(hi, ri[:2000])
    np.testing.assert_array_equal(hd, rd[:2000])


def test_c1_restatement_counters_per_query(c1, gpu):
    """Per query (not only in total), the device's six counters equal the
    restatement's at ef = 64."""
    import torch
    base, queries, path = c1
    g = oracle.OraGraph.load(path)
    oi, od, ocnt = g.search(queries, K, 64, counters=True)
    idx = HNSWIndex.load(path)
    q = torch.from_numpy(queries).cuda()
    ids = torch.empty((NQ, K), dtype=torch.int32, device="cuda")
    ds = torch.empty((NQ, K), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((NQ, 6), dtype=torch.int32, device="cuda")
    idx.search_device(q, K, 64, ids, ds, counters=cnt)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ids.cpu().numpy(), oi)
    np.testing.assert_array_equal(ds.cpu().numpy(), od)
    np.testing.assert_array_equal(cnt.cpu().numpy(), ocnt.astype(np.int32))
