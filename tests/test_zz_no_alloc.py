"""pk_index_search_noalloc: the exact device search for callers that cannot
let a library allocate device memory (a latency-critical serving loop that
must not take cudaMalloc's implicit synchronisation, or a process whose device
memory another allocator already owns).  Its scratch is a fixed array inside
the library; the test calls it through the C ABI twice in a row and checks
both answers against pk_index_search_device, and checks that requests beyond
its stated limits are refused with a clear error.

This file is collected last on purpose, so that a run stopping at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

import oracle
from pickle_b200 import HNSWIndex, datasets, lib
from tests.helpers import case_data, ref_graph

pytestmark = pytest.mark.gpu


def _bind():
    L = lib()
    f = L.pk_index_search_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return L, f


def _call(idx, q, k, ef, ids, ds):
    _, f = _bind()
    return f(idx._h, ctypes.c_void_p(q.data_ptr()), q.shape[0], k, ef, ctypes.c_void_p(ids.data_ptr()),
             ctypes.c_void_p(ds.data_ptr()), None)


# u8_l2: rows already 16-byte multiples; i8_l2_d100: rows of 100 bytes are
# staged into the fixed array; f32unit_ip: float data, inner product
@pytest.mark.parametrize("name", ["u8_l2", "i8_l2_d100", "f32unit_ip"])
def test_noalloc_search_equals_device_search_on_two_calls(name, gpu, ref_bin):
    import torch
    metric, base, queries, M, efc = case_data(name)
    idx = HNSWIndex.load(ref_graph(name))
    q = torch.from_numpy(queries).cuda()
    k, ef = 10, 40
    want_ids = torch.empty((len(queries), k), dtype=torch.int32, device="cuda")
    want_ds = torch.empty((len(queries), k), dtype=torch.float32, device="cuda")
    idx.search_device(q, k, ef, want_ids, want_ds)
    torch.cuda.synchronize()
    for _ in range(2):
        ids = torch.full((len(queries), k), -7, dtype=torch.int32, device="cuda")
        ds = torch.zeros((len(queries), k), dtype=torch.float32, device="cuda")
        rc = _call(idx, q, k, ef, ids, ds)
        assert rc == 0, lib().pk_last_error()
        torch.cuda.synchronize()
        # the same kernel on the same data: identical, the tests' tolerance for
        # any path that keeps the reference's heap order
        np.testing.assert_array_equal(ids.cpu().numpy(), want_ids.cpu().numpy())
        np.testing.assert_array_equal(ds.cpu().numpy(), want_ds.cpu().numpy())


def _want(idx, q, k, ef):
    import torch
    ids = torch.empty((q.shape[0], k), dtype=torch.int32, device="cuda")
    ds = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    idx.search_device(q, k, ef, ids, ds)
    torch.cuda.synchronize()
    return ids.cpu().numpy(), ds.cpu().numpy()


def _got(idx, q, k, ef):
    import torch
    ids = torch.full((q.shape[0], k), -7, dtype=torch.int32, device="cuda")
    ds = torch.zeros((q.shape[0], k), dtype=torch.float32, device="cuda")
    rc = _call(idx, q, k, ef, ids, ds)
    assert rc == 0, lib().pk_last_error()
    torch.cuda.synchronize()
    return ids.cpu().numpy(), ds.cpu().numpy()


def test_noalloc_sequence_of_shapes_and_indexes(gpu, ref_bin):
    """The fixed array keeps each call's leftovers: a few queries (few warps,
    a small bitmap area), the whole batch (more warps: the bitmap area grows
    over memory the previous call used for lists and spills), an index with a
    larger layer 0 (larger bitmaps), then the first call again.  Every answer
    equals pk_index_search_device's, and on integer data the oracle's."""
    import torch
    metric, base, queries, M, efc = case_data("u8_l2")
    path = ref_graph("u8_l2")
    a = HNSWIndex.load(path)
    qa = torch.from_numpy(queries).cuda()
    big_base, big_q = datasets.gmm_bytes(12000, 300, 64, ncomp=16, seed=5)
    b = HNSWIndex(64, np.uint8, "l2", M=8, ef_construction=64)
    b.set_seed(5)
    b.build(big_base)
    qb = torch.from_numpy(big_q).cuda()
    oi, od = oracle.OraGraph.load(path).search(queries, 10, 40)
    for idx, q, k, ef in [(a, qa[:4], 10, 40), (a, qa, 10, 40), (b, qb, 16, 200), (b, qb[:7], 5, 64),
                          (a, qa[:4], 10, 40), (a, qa, 10, 40)]:
        gi, gd = _got(idx, q, k, ef)
        wi, wd = _want(idx, q, k, ef)
        np.testing.assert_array_equal(gi, wi)
        np.testing.assert_array_equal(gd, wd)
        if idx is a:
            np.testing.assert_array_equal(gi, oi[:q.shape[0]])
            np.testing.assert_array_equal(gd, od[:q.shape[0]])


def test_noalloc_refuses_requests_beyond_its_limits(gpu, ref_bin):
    import torch
    metric, base, queries, M, efc = case_data("u8_l2")
    idx = HNSWIndex.load(ref_graph("u8_l2"))
    q = torch.from_numpy(queries).cuda()
    ids = torch.empty((len(queries), 10), dtype=torch.int32, device="cuda")
    ds = torch.empty((len(queries), 10), dtype=torch.float32, device="cuda")
    assert _call(idx, q, 10, 5000, ids, ds) == -1
    assert b"1024" in lib().pk_last_error()
    big = torch.zeros((65537, queries.shape[1]), dtype=torch.uint8, device="cuda")
    bids = torch.empty((65537, 1), dtype=torch.int32, device="cuda")
    bds = torch.empty((65537, 1), dtype=torch.float32, device="cuda")
    assert _call(idx, big, 1, 16, bids, bds) == -1
    assert b"65536" in lib().pk_last_error()
