"""Pins of the oracle (oracle/pk_oracle.c, the C restatement) against the
reference's own code: live against oracle/_ref/pk_ref where it is built, and
against the committed golden fixtures (tests/golden, made by pk_ref) always.
CPU only."""
import json
import os

import numpy as np
import pytest

import oracle
from tests.helpers import (CASES, INTEGER_CASES, case_data, compare_float_results, mismatched_queries, ref_graph,
                           reference_distance_table)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = ["f32int_l2", "u8_ip", "i8_l2_d100", "f16_ip"]


# ------------------------------------------------------------ distances ----

def test_distance_known_answers():
    a = np.arange(1, 33, dtype=np.uint8)
    b = np.arange(32, 0, -1).astype(np.uint8)
    assert oracle.distance("l2", a, b) == float(((a.astype(int) - b) ** 2).sum())
    assert oracle.distance("ip", a, b) == -float((a.astype(int) * b).sum())
    s = np.array([-128, 127, -1, 5] * 25, np.int8)
    t = np.array([127, -128, 3, -5] * 25, np.int8)
    assert oracle.distance("l2", s, t) == float(((s.astype(int) - t) ** 2).sum())
    assert oracle.distance("ip", s, t) == -float((s.astype(int) * t).sum())
    x = np.full(96, 2.0, np.float32)
    assert oracle.distance("l2", x, np.zeros(96, np.float32)) == 384.0
    assert oracle.distance("ip", x, x) == -384.0


@pytest.mark.parametrize("dtype", [np.uint8, np.int8])
@pytest.mark.parametrize("dim", [32, 96, 100, 128, 768])
def test_integer_distances_bit_exact_vs_reference(dtype, dim, ref_bin):
    rng = np.random.default_rng(dim)
    info = np.iinfo(dtype)
    a = rng.integers(info.min, info.max + 1, size=(200, dim)).astype(dtype)
    b = rng.integers(info.min, info.max + 1, size=(200, dim)).astype(dtype)
    for metric in ("l2", "ip"):
        ref = oracle.ref_dist(metric, a, b)
        mine = np.array([oracle.distance(metric, a[i], b[i]) for i in range(len(a))], np.float32)
        np.testing.assert_array_equal(mine, ref)


@pytest.mark.parametrize("dtype", [np.float32, np.float16])
@pytest.mark.parametrize("dim", [96, 128, 768])
def test_float_distances_close_to_reference(dtype, dim, ref_bin):
    """The reference's float sums are reassociated by its compiler; the
    restatement uses the source order: they agree to rounding."""
    rng = np.random.default_rng(dim)
    a = rng.normal(size=(200, dim)).astype(dtype)
    b = rng.normal(size=(200, dim)).astype(dtype)
    for metric in ("l2", "ip"):
        ref = oracle.ref_dist(metric, a, b).astype(np.float64)
        mine = np.array([oracle.distance(metric, a[i], b[i]) for i in range(len(a))], np.float64)
        scale = (np.abs(a.astype(np.float64)) * np.abs(b.astype(np.float64))).sum(1) + \
            ((a.astype(np.float64) - b) ** 2).sum(1)
        assert (np.abs(ref - mine) <= 1e-5 * scale).all()


# --------------------------------------------------------------- search ----

@pytest.mark.parametrize("name", sorted(CASES))
def test_search_restatement_matches_reference(name, ref_bin):
    metric, base, queries, M, efc = case_data(name)
    path = ref_graph(name)
    ri, rd, info = oracle.ref_search(path, queries, 10, 32, threads=4, metrics=True)
    g = oracle.OraGraph.load(path)
    oi, od, cnt = g.search(queries, 10, 32, threads=4, counters=True)
    if name in INTEGER_CASES:
        np.testing.assert_array_equal(oi, ri)
        np.testing.assert_array_equal(od, rd)
        assert cnt[:, 0].sum() + cnt[:, 3].sum() == info["hop"]
        assert cnt[:, 1].sum() + cnt[:, 4].sum() == info["dist"]
        assert cnt[:, 3].sum() == info["base_hop"]
        assert cnt[:, 4].sum() == info["base_dist"]
        assert cnt[:, 2].sum() + cnt[:, 5].sum() == info["neighbor"]
    else:
        # float sums are rounded differently by the reference's compiler:
        # wherever the two sets of distances never disagree on a comparison
        # the results must be the reference's; see the fork test below
        assert len(mismatched_queries(oi, od, ri, rd)) <= 0.05 * len(queries)


@pytest.mark.parametrize("name", sorted(set(CASES) - INTEGER_CASES))
def test_float_search_forks_only_at_near_ties(name, ref_bin):
    """The restatement replayed with the reference binary's own distances
    (pk_ref dist, the instantiation its search runs) compared at every
    decision: a query whose decisions never flip returns the reference's ids,
    and every query whose ids differ from the reference's beyond 1e-6 ties
    flips first at a comparison of two distances within 1e-6 of each other."""
    metric, base, queries, M, efc = case_data(name)
    path = ref_graph(name)
    ri, rd, _ = oracle.ref_search(path, queries, 10, 32, threads=4)
    g = oracle.OraGraph.load(path)
    oi, od = g.search(queries, 10, 32, threads=4)
    _, _, _, touched = g.search_fork(queries, 10, 32, oracle.ORDER_SOURCE, oracle.ORDER_SOURCE, threads=4,
                                     touched_cap=100_000)
    table = reference_distance_table(base, queries, touched, metric)
    fi, fd, fork, _ = g.search_fork(queries, 10, 32, oracle.ORDER_SOURCE, oracle.ORDER_TABLE, table=table, threads=4)
    np.testing.assert_array_equal(fi, oi)
    np.testing.assert_array_equal(fd, od)
    assert (fork[:, 1] != 5).all()
    calm = fork[:, 0] == 0
    np.testing.assert_array_equal(oi[calm], ri[calm])
    for qi in mismatched_queries(oi, od, ri, rd):
        f = fork[qi]
        assert f[0] == 1.0
        gap_a = abs(f[2] - f[3]) / max(abs(f[2]), abs(f[3]))
        gap_b = abs(f[4] - f[5]) / max(abs(f[4]), abs(f[5]))
        assert min(gap_a, gap_b) <= 1e-6, (qi, f)


def test_fork_detector_consistency():
    """Same order on both sides: no fork and the plain search's results; a
    table holding the driving order's own distances: no fork either."""
    metric, base, queries, M, efc = case_data("f32unit_ip")
    path = ref_graph("f32unit_ip")
    g = oracle.OraGraph.load(path)
    for order in (oracle.ORDER_SOURCE, oracle.ORDER_DEVICE):
        with oracle.float_order(order):
            oi, od = g.search(queries, 10, 40, threads=4)
        fi, fd, fork, touched = g.search_fork(queries, 10, 40, order, order, threads=4, touched_cap=100_000)
        np.testing.assert_array_equal(fi, oi)
        np.testing.assert_array_equal(fd, od)
        assert (fork[:, 0] == 0).all()
        keys = [np.unique(t) for t in touched]
        off = np.zeros(len(keys) + 1, np.int64)
        off[1:] = np.cumsum([len(x) for x in keys])
        K = np.concatenate(keys).astype(np.int32)
        qi = np.repeat(np.arange(len(keys)), [len(x) for x in keys])
        with oracle.float_order(order):
            vals = np.array([oracle.distance(metric, queries[i], base[k] if k >= 0 else np.zeros_like(base[0]))
                             for i, k in zip(qi, K)], np.float32)
        _, _, fork, _ = g.search_fork(queries, 10, 40, order, oracle.ORDER_TABLE, table=(off, K, vals), threads=4)
        assert (fork[:, 0] == 0).all()
    # the two orders do disagree somewhere, and where the results differ the
    # search forked
    with oracle.float_order(oracle.ORDER_DEVICE):
        di, dd = g.search(queries, 10, 40, threads=4)
    si, sd = g.search(queries, 10, 40, threads=4)
    _, _, fork, _ = g.search_fork(queries, 10, 40, oracle.ORDER_DEVICE, oracle.ORDER_SOURCE, threads=4)
    for q in np.nonzero((di != si).any(1))[0]:
        assert fork[q, 0] == 1.0


def test_device_order_distances():
    """The device order's distances are float32 roundings of the exact value:
    integer-valued rows give the exact integer, others agree with float64 to
    a few units in the last place."""
    rng = np.random.default_rng(4)
    for dim in (32, 48, 96, 100, 128, 768):
        ai = rng.integers(0, 256, size=(50, dim)).astype(np.float32)
        bi = rng.integers(0, 256, size=(50, dim)).astype(np.float32)
        af = rng.normal(size=(50, dim)).astype(np.float32)
        bf = rng.normal(size=(50, dim)).astype(np.float32)
        with oracle.float_order(oracle.ORDER_DEVICE):
            for i in range(50):
                assert oracle.distance("l2", ai[i], bi[i]) == float(((ai[i].astype(np.int64) - bi[i]) ** 2).sum())
                for metric, exact in (("l2", ((af[i].astype(np.float64) - bf[i]) ** 2).sum()),
                                      ("ip", -(af[i].astype(np.float64) * bf[i]).sum())):
                    scale = (np.abs(af[i].astype(np.float64)) * np.abs(bf[i]) + (af[i].astype(np.float64) - bf[i]) ** 2).sum()
                    assert abs(oracle.distance(metric, af[i], bf[i]) - exact) <= 1e-6 * scale
                for dt in (np.float16,):
                    x, y = af[i].astype(dt), bf[i].astype(dt)
                    ex = ((x.astype(np.float64) - y) ** 2).sum()
                    assert abs(oracle.distance("l2", x, y) - ex) <= 1e-6 * ex


@pytest.mark.parametrize("name", ["f32int_l2", "u8_ip", "i8_l2_d100", "i8_ip"])
def test_build_restatement_matches_reference_byte_for_byte(name, ref_bin, tmp_path):
    metric, base, queries, M, efc = case_data(name)
    n = 2500
    base = base[:n]
    order = np.random.default_rng(9).permutation(n).astype(np.int32)
    from tests.helpers import levels_for
    lv = levels_for(n, M, 9)
    rp, op = str(tmp_path / "ref.pkg"), str(tmp_path / "ora.pkg")
    info = oracle.ref_build(base, metric, M, efc, rp, threads=1, order=order, levels=lv)
    g = oracle.OraGraph.new(metric, base.dtype, base.shape[1], M, efc, lv, oracle.GROWTH_REFERENCE)
    g.build(base, order)
    g.save(op)
    assert open(rp, "rb").read() == open(op, "rb").read()
    assert info["degree_over_cap"] >= 0


def test_reference_lists_outgrow_their_cap(ref_bin, tmp_path):
    """The reference's AddEdge re-prune appends without a bound
    (include/hnsw_layer.hpp:441-447); the capped growth mode does not."""
    metric, base, queries, M, efc = case_data("f32int_l2")
    from tests.helpers import levels_for
    n = len(base)
    order = np.arange(n, dtype=np.int32)
    lv = levels_for(n, M, 1)
    info = oracle.ref_build(base, metric, M, efc, str(tmp_path / "r.pkg"), threads=1, order=order, levels=lv)
    assert info["degree_over_cap"] > 0
    g = oracle.OraGraph.new(metric, base.dtype, base.shape[1], M, efc, lv, oracle.GROWTH_CAPPED)
    g.build(base, order)
    for level in range(g.info()["num_layers"]):
        L = g.layer(level)
        assert (L["degree"] <= L["cap"]).all()


# --------------------------------------------------------------- golden ----

@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_build_and_search(name, tmp_path):
    """Without running the reference: its recorded Build output and search
    results, reproduced by the restatement."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    data, order, levels, queries = z["data"], z["order"], z["levels"], z["queries"]
    g = oracle.OraGraph.new(meta["metric"], data.dtype, data.shape[1], meta["M"], meta["efc"], levels,
                            oracle.GROWTH_REFERENCE)
    g.build(data, order)
    out = str(tmp_path / "g.pkg")
    g.save(out)
    golden_pkg = os.path.join(GOLDEN, name + ".pkg")
    if data.dtype != np.float16:
        assert open(out, "rb").read() == open(golden_pkg, "rb").read()
    ref = oracle.OraGraph.load(golden_pkg)
    oi, od, cnt = ref.search(queries, meta["k"], meta["ef"], counters=True)
    if data.dtype != np.float16:
        np.testing.assert_array_equal(oi, z["ids"])
        np.testing.assert_array_equal(od, z["dists"])
        assert cnt[:, 1].sum() + cnt[:, 4].sum() == meta["counters"]["dist"]
    else:
        assert compare_float_results(oi, od, z["ids"], z["dists"]) >= 0.95


def test_graph_file_roundtrip_and_corruption(tmp_path):
    src = os.path.join(GOLDEN, "u8_ip.pkg")
    g = oracle.OraGraph.load(src)
    out = str(tmp_path / "copy.pkg")
    g.save(out)
    assert open(out, "rb").read() == open(src, "rb").read()
    raw = bytearray(open(src, "rb").read())
    raw[len(raw) // 2] ^= 0x40
    bad = str(tmp_path / "bad.pkg")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(IOError):
        oracle.OraGraph.load(bad)
    open(bad, "wb").write(bytes(raw[: len(raw) // 3]))
    with pytest.raises(IOError):
        oracle.OraGraph.load(bad)


def test_level_distribution_formula():
    for M in (4, 8, 16, 32, 48):
        cp = oracle.cumulative_probability(M)
        r = 1.0 / np.log(M)
        want = np.cumsum([np.exp(-l / r) * (1 - np.exp(-1 / r)) for l in range(len(cp))])
        np.testing.assert_allclose(cp, want, rtol=1e-12)
        assert np.exp(-len(cp) / r) * (1 - np.exp(-1 / r)) < 1e-9


def v2_checksum(payload: bytes) -> int:
    """The version 2 graph-file checksum, restated from its definition: 4 MiB
    blocks, each digested as FNV-1a 64 over little-endian 64-bit words (last
    word zero padded) and then its length; FNV-1a 64 over the digests, then
    the total length."""
    P, B, M = 1099511628211, 4 << 20, (1 << 64) - 1
    h = 1469598103934665603
    for b0 in range(0, len(payload), B):
        blk = payload[b0:b0 + B]
        pad = blk + b"\0" * (-len(blk) % 8)
        d = 1469598103934665603
        for w in np.frombuffer(pad, "<u8").tolist():
            d = ((d ^ w) * P) & M
        d = ((d ^ len(blk)) * P) & M
        h = ((h ^ d) * P) & M
    return ((h ^ len(payload)) * P) & M


def test_graph_file_version_2_block_checksum(tmp_path):
    """A version 2 file (the device library's format: block checksum) is read
    by the oracle like the version 1 file it was made from; a flipped byte
    is caught."""
    src = open(os.path.join(GOLDEN, "u8_ip.pkg"), "rb").read()
    body = bytearray(src[:-8])
    body[8:12] = (2).to_bytes(4, "little")
    v2 = bytes(body) + v2_checksum(bytes(body)).to_bytes(8, "little")
    p = str(tmp_path / "v2.pkg")
    open(p, "wb").write(v2)
    z = np.load(os.path.join(GOLDEN, "u8_ip.npz"))
    meta = json.loads(str(z["meta"]))
    a = oracle.OraGraph.load(os.path.join(GOLDEN, "u8_ip.pkg")).search(z["queries"], meta["k"], meta["ef"])
    b = oracle.OraGraph.load(p).search(z["queries"], meta["k"], meta["ef"])
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    bad = bytearray(v2)
    bad[len(bad) // 3] ^= 1
    open(p, "wb").write(bytes(bad))
    with pytest.raises(IOError):
        oracle.OraGraph.load(p)
