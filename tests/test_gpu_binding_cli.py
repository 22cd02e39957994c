"""The Python binding in the reference binding's shape (pybind/hnsw.cpp:116-127)
and the command-line driver in the reference benchmark's shape
(benchmark/hnsw_pickle.cpp:64-122, benchmark/bench_util.hpp:24-25)."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from pickle_b200 import HNSWIndex, datasets

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_binding_properties_build_search_save_load(gpu, tmp_path):
    base, queries = datasets.gmm_int_f32(3000, 100, 32, ncomp=16, seed=2)
    idx = HNSWIndex()
    assert (idx.search_ef, idx.build_ef, idx.top_k, idx.M, idx.num_layer) == (100, 100, 10, 32, 0)
    idx.M = 8
    idx.build_ef = 64
    idx.top_k = 5
    idx.search_ef = 40
    idx.build(base)
    info = idx.info()
    assert info["M"] == 8 and info["ef_construction"] == 64 and info["n"] == 3000
    assert idx.num_layer == info["num_layers"] >= 1
    ids = idx.search(queries)
    assert ids.shape == (100, 5) and ids.dtype == np.int32
    ri, rd = idx.search(queries, 5, 40)
    np.testing.assert_array_equal(ids, ri)
    p = str(tmp_path / "g.pkg")
    idx.save(p)
    other = HNSWIndex()
    other.top_k, other.search_ef = 5, 40
    assert other.load(p) is other
    np.testing.assert_array_equal(other.search(queries), ids)
    np.testing.assert_array_equal(HNSWIndex.load(p).search(queries, 5, 40)[0], ids)
    # a second build replaces the index, as the reference binding's does
    idx.M = 12
    idx.build(base[:1500])
    assert idx.info()["n"] == 1500 and idx.info()["M"] == 12
    fixed = HNSWIndex(32, np.float32, "l2", M=8, ef_construction=64)
    with pytest.raises(ValueError):
        fixed.M = 16


def test_per_query_host_searches_equal_uniform_ones(gpu):
    base, queries = datasets.gmm_int_f32(3000, 60, 32, ncomp=16, seed=3)
    idx = HNSWIndex(32, np.float32, "l2", M=8, ef_construction=64)
    idx.set_seed(3)
    idx.build(base)
    idx.prepare_fast("f16")
    rng = np.random.default_rng(4)
    kq = rng.choice([1, 5, 10], size=len(queries)).astype(np.int32)
    efq = rng.integers(10, 90, size=len(queries)).astype(np.int32)
    for var, one in ((idx.search_var, idx.search), (idx.search_fast_var, idx.search_fast)):
        ids, ds = var(queries, kq, efq)
        assert ids.shape == (len(queries), 10)
        for i in range(len(queries)):
            ui, ud = one(queries[i:i + 1], int(kq[i]), int(efq[i]))
            np.testing.assert_array_equal(ids[i, :kq[i]], ui[0])
            np.testing.assert_array_equal(ds[i, :kq[i]], ud[0])
            assert (ids[i, kq[i]:] == -1).all()


LINE = re.compile(r"^k=(\d+) search_ef=(\d+) recall=([\d.]+|nan) qps/t=(\d+) hop=([\d.]+) dist=([\d.]+) "
                  r"base_hop=([\d.]+) base_dist=([\d.]+) build_ef=(\d+) thread=(\d+)$")


def _cli(*args):
    p = subprocess.run([sys.executable, "-m", "pickle_b200.cli"] + [str(a) for a in args], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


def test_cli_build_search_log_lines(gpu, tmp_path):
    d = tmp_path / "data"
    _cli("gen", "--config", "c1", "--n", 3000, "--nq", 40, "--out", d, "--labels")
    g, log = tmp_path / "g.pkg", tmp_path / "log.txt"
    _cli("build", "--feat_path", d / "feat.npy", "--space", "l2", "--max_degree", 8, "--build_ef", 64,
         "--index_path", g, "--log_path", log)
    out_ids = tmp_path / "ids.npy"
    _cli("search", "--index_path", g, "--query_path", d / "query.npy", "--label_path", d / "label.npy",
         "--k", 10, "--ef", 48, "--repeat", 1, "--log_path", log, "--out_ids", out_ids)
    lines = open(log).read().strip().split("\n")
    assert lines[0].startswith("BuildTime=")
    m = LINE.match(lines[1])
    assert m, lines[1]
    assert (int(m.group(1)), int(m.group(2)), int(m.group(9)), int(m.group(10))) == (10, 48, 64, 1)
    q = np.load(d / "query.npy")
    labels = np.load(d / "label.npy")
    want, _ = HNSWIndex.load(str(g)).search(q, 10, 48)
    got = np.load(out_ids)
    np.testing.assert_array_equal(got, want)
    assert float(m.group(3)) == round(100.0 * datasets.recall_at_k(want, labels, 10), 1)
    assert float(m.group(5)) >= float(m.group(7)) > 0 and float(m.group(6)) >= float(m.group(8)) > 0
    # without --k/--ef: the reference's grid, k in {1, 10, 100} x ef in
    # {1, ..., 500}, skipping ef < k
    sweep = _cli("search", "--index_path", g, "--query_path", d / "query.npy", "--repeat", 1, "--no_metrics")
    pairs = [(int(x.group(1)), int(x.group(2))) for x in map(LINE.match, sweep.strip().split("\n")) if x]
    grid = [1, 5, 10, 20, 30, 50, 70, 90, 100, 200, 300, 400, 500]
    assert pairs == [(k, e) for k in (1, 10, 100) for e in grid if e >= k]
