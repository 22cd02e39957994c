"""The header-only C++ front end (include/pickle_b200/hnsw.hpp) compiles
against the C ABI, links with the library, and on a GPU builds, searches and
round-trips an index; without a GPU it reports the no-device status."""
import os
import subprocess

import pytest

import pickle_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "hnsw_api_demo")
    src = os.path.join(ROOT, "tests", "cpp", "hnsw_api_demo.cpp")
    libdir = os.path.dirname(pickle_b200.LIB_PATH)
    subprocess.run(["g++", "-std=c++20", "-O1", "-I" + os.path.join(ROOT, "include"), src, "-o", exe,
                    "-L" + libdir, "-l:libpickle_b200.so", "-Wl,-rpath," + libdir], check=True)
    return exe


def test_cpp_front_end_compiles_and_reports_status(tmp_path):
    import torch
    exe = _build(tmp_path)
    p = subprocess.run([exe, str(tmp_path / "g.pkg")], capture_output=True, text=True, timeout=300)
    if torch.cuda.is_available():
        assert p.returncode == 0, p.stdout + p.stderr
    else:
        assert p.returncode == 3 and "error -9" in p.stdout, p.stdout


@pytest.mark.gpu
def test_cpp_front_end_on_gpu(tmp_path, gpu):
    exe = _build(tmp_path)
    p = subprocess.run([exe, str(tmp_path / "g.pkg")], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    first = p.stdout.split("\n")[0].split()
    assert first[0] == "ids" and first[1] == "0"  # the query is row 0 itself
    assert "reload same" in p.stdout
