"""Continuous batching (pk_server_*): requests with mixed k and ef, submitted
while others are on the GPU, are packed into free slots, overlap on the
device, and each result equals the one the same request gets alone.
Failure handling is tested on the host: an expired watchdog fails requests
with PK_ERR_TIMEOUT, requests beyond the server's limits are refused."""
import threading

import numpy as np
import pytest

from pickle_b200 import HNSWIndex, PickleError, Server, datasets
from tests.helpers import case_data, ref_graph

pytestmark = pytest.mark.gpu


def _index():
    idx = HNSWIndex.load(ref_graph("f32unit_ip"))
    idx.prepare_fast("f16")
    return idx


def test_each_result_equals_alone_in_the_mix(gpu, ref_bin):
    metric, base, queries, M, efc = case_data("f32unit_ip")
    idx = _index()
    rng = np.random.default_rng(8)
    reqs = []
    for _ in range(60):
        nq = int(rng.integers(1, 40))
        sel = rng.integers(0, len(queries), size=nq)
        k = int(rng.choice([1, 5, 10, 20]))
        ef = int(rng.integers(max(k, 16), 120))
        reqs.append((queries[sel], k, ef))
    srv = Server(idx, "f16", slots=3, max_batch=256, max_k=20, max_ef=128)
    tickets = [None] * len(reqs)

    def producer(lo, hi):
        for i in range(lo, hi):
            tickets[i] = srv.submit(*reqs[i])

    ths = [threading.Thread(target=producer, args=(i * 20, i * 20 + 20)) for i in range(3)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for i, (q, k, ef) in enumerate(reqs):
        ids, ds, lat = srv.wait(tickets[i])
        ai, ad = idx.search_fast(q, k, ef)
        np.testing.assert_array_equal(ids, ai)
        np.testing.assert_array_equal(ds, ad)
        assert lat >= 0
    st = srv.stats()
    assert st["queries"] >= sum(len(r[0]) for r in reqs) and st["error"] == 0
    assert st["batches"] >= 2
    srv.close()


def test_slots_overlap_under_load(gpu, ref_bin):
    metric, base, queries, M, efc = case_data("f32unit_ip")
    idx = _index()
    srv = Server(idx, "f16", slots=4, max_batch=64, max_k=10, max_ef=64)
    ts = [srv.submit(queries[(i * 50) % 150:(i * 50) % 150 + 50], 10, 64) for i in range(40)]
    for t in ts:
        srv.wait(t)
    assert srv.stats()["max_inflight"] >= 2
    srv.close()


def test_limits_and_watchdog(gpu, ref_bin):
    metric, base, queries, M, efc = case_data("f32unit_ip")
    idx = _index()
    srv = Server(idx, "f16", slots=2, max_batch=32, max_k=10, max_ef=64)
    with pytest.raises(PickleError):
        srv.submit(queries[:64], 10, 32)      # more queries than a batch holds
    with pytest.raises(PickleError):
        srv.submit(queries[:4], 11, 32)       # k beyond max_k
    # a watchdog of 0 s expires for any batch still in flight when polled
    srv.set_watchdog(0.0)
    t = srv.submit(queries[:32], 10, 64)
    with pytest.raises(PickleError) as e:
        srv.wait(t, timeout_ms=10000)
    assert e.value.code in (-7,)
    srv.close()
