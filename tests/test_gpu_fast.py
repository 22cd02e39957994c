"""The batched low-precision search (FP16 or per-dimension-scaled FP8
traversal, exact re-rank).  Judged by recall, as the reference's own search
is the exact path: its recall@10 must stay within a stated margin of the
exact path's at the same ef, its returned distances must be the exact
distances of the returned ids, rows must be ascending with no repeated ids,
and a mixed-k/ef launch must answer each query as a uniform launch does."""
import numpy as np
import pytest

import oracle
from pickle_b200 import HNSWIndex, datasets
from tests.helpers import CASES, INTEGER_CASES, case_data, ref_graph

pytestmark = pytest.mark.gpu

# FP16 walks as well as the exact path at the same ef (recall@10 within 0.01);
# FP8 E4M3 (3 mantissa bits) reorders the walk more and needs a larger list:
# at 3x the ef it must reach the exact path's recall within 0.02
EF_FACTOR = {"f16": 1, "fp8": 3}
MARGIN = {"f16": 0.01, "fp8": 0.02}


@pytest.mark.parametrize("trav", ["f16", "fp8"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fast_recall_and_exact_distances(name, trav, gpu, ref_bin):
    metric, base, queries, M, efc = case_data(name)
    idx = HNSWIndex.load(ref_graph(name))
    idx.prepare_fast(trav)
    k, ef = 10, 48
    gt, _ = datasets.exact_knn(base, queries, k, metric)
    ei, ed = idx.search(queries, k, ef)
    fi, fd = idx.search_fast(queries, k, ef * EF_FACTOR[trav])
    r_exact = datasets.recall_at_k(ei, gt, k)
    r_fast = datasets.recall_at_k(fi, gt, k)
    assert r_fast >= r_exact - MARGIN[trav], (r_fast, r_exact)
    # ascending, no repeats, padded only at the end
    for row_i, row_d in zip(fi, fd):
        valid = row_i >= 0
        assert (np.diff(row_d[valid]) >= 0).all()
        assert len(set(row_i[valid].tolist())) == valid.sum()
    # distances are the exact ones of the returned ids
    for qi in range(0, len(queries), 17):
        for j in range(k):
            if fi[qi, j] < 0:
                continue
            want = oracle.distance(metric, queries[qi], base[fi[qi, j]])
            if name in INTEGER_CASES:
                assert fd[qi, j] == want
            else:
                assert abs(fd[qi, j] - want) <= 1e-4 * max(1.0, abs(want))


@pytest.mark.parametrize("trav", ["f16", "fp8"])
def test_fast_mixed_k_ef_equals_uniform(trav, gpu, ref_bin):
    import torch
    metric, base, queries, M, efc = case_data("f32unit_ip")
    idx = HNSWIndex.load(ref_graph("f32unit_ip"))
    idx.prepare_fast(trav)
    rng = np.random.default_rng(4)
    nq = len(queries)
    ks = rng.choice([1, 10, 20], size=nq).astype(np.int32)
    efs = rng.integers(20, 130, size=nq).astype(np.int32)
    stride = int(ks.max())
    q = torch.from_numpy(queries).cuda()
    ids = torch.full((nq, stride), -7, dtype=torch.int32, device="cuda")
    ds = torch.zeros((nq, stride), dtype=torch.float32, device="cuda")
    idx.search_fast_device(q, stride, int(efs.max()), ids, ds, k_per_query=torch.from_numpy(ks).cuda(),
                           ef_per_query=torch.from_numpy(efs).cuda())
    torch.cuda.synchronize()
    ids, ds = ids.cpu().numpy(), ds.cpu().numpy()
    for i in range(0, nq, 9):
        ui, ud = idx.search_fast(queries[i:i + 1], int(ks[i]), int(efs[i]))
        np.testing.assert_array_equal(ids[i, :ks[i]], ui[0])
        np.testing.assert_array_equal(ds[i, :ks[i]], ud[0])


def test_fast_after_insert_covers_new_rows(gpu):
    """Rows added after prepare_fast are converted with the same scales."""
    base, queries = datasets.gmm_unit(3000, 100, 32, ncomp=16, seed=5)
    idx = HNSWIndex(32, np.float32, "ip", M=8, ef_construction=64)
    idx.build(base[:2000])
    idx.prepare_fast("fp8")
    idx.add(base[2000:], np.arange(2000, 3000, dtype=np.int32))
    gt, _ = datasets.exact_knn(base, queries, 10, "ip")
    fi, _ = idx.search_fast(queries, 10, 64)
    assert datasets.recall_at_k(fi, gt, 10) >= 0.9
    assert (fi >= 2000).any()
