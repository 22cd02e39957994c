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


def test_admission_waits_for_device_memory_not_for_slots(gpu, ref_bin):
    """Eight free slots, but device memory for about one request at a time:
    the requests are served one after another (never two batches in flight),
    the waiting ones are counted as deferred for memory, each result is the
    one the request gets alone, and a request larger than the whole arena is
    refused at submission."""
    metric, base, queries, M, efc = case_data("f32unit_ip")
    idx = _index()
    probe = Server(idx, "f16", slots=1, max_batch=256, max_k=10, max_ef=128)
    one = probe.request_bytes(150, 10, 128)
    assert probe.request_bytes(300, 10, 128) > one and probe.request_bytes(150, 10, 64) < one
    probe.close()
    srv = Server(idx, "f16", slots=8, max_batch=512, max_k=10, max_ef=128, device_bytes=int(one * 1.5))
    reqs = [queries[(i * 37) % 50:(i * 37) % 50 + 150] for i in range(6)]
    ts = [srv.submit(q, 10, 128) for q in reqs]
    for q, t in zip(reqs, ts):
        ids, ds, _ = srv.wait(t)
        ai, ad = idx.search_fast(q, 10, 128)
        np.testing.assert_array_equal(ids, ai)
        np.testing.assert_array_equal(ds, ad)
    st, mem = srv.stats(), srv.memory()
    assert st["max_inflight"] == 1 and st["batches"] == 6, st
    assert mem["deferred_for_memory"] >= 1 and mem["in_use"] == 0, mem
    assert one <= mem["peak_in_use"] <= mem["arena_bytes"], mem
    with pytest.raises(PickleError) as e:
        srv.submit(np.concatenate([queries, queries])[:400], 10, 128)
    assert e.value.code == -10
    srv.close()


def test_ef_up_to_1024(gpu, ref_bin):
    """The fast path takes ef up to 1024 (list widths 24 and 32 slots per
    lane); its distances are the exact ones and its recall at ef 1024 is at
    least that at ef 512; a server takes such requests too."""
    import oracle
    metric, base, queries, M, efc = case_data("f32unit_ip")
    idx = _index()
    gt, _ = datasets.exact_knn(base, queries, 10, metric)
    i5, _ = idx.search_fast(queries, 10, 512)
    i10, d10 = idx.search_fast(queries, 10, 1024)
    assert datasets.recall_at_k(i10, gt, 10) >= datasets.recall_at_k(i5, gt, 10) - 1e-9
    want = np.array([[oracle.distance(metric, q, base[j]) for j in row] for q, row in zip(queries, i10)], np.float32)
    np.testing.assert_allclose(d10, want, rtol=2e-6, atol=1e-6)
    srv = Server(idx, "f16", slots=2, max_batch=64, max_k=10, max_ef=1024)
    t = srv.submit(queries[:40], 10, 1000)
    ids, ds, _ = srv.wait(t)
    ai, ad = idx.search_fast(queries[:40], 10, 1000)
    np.testing.assert_array_equal(ids, ai)
    srv.close()
