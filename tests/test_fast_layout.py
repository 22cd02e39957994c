"""The fast walk's launch arithmetic (pickle_b200/csrc/pk_fast.h), checked on the
CPU: list-width classes for every ef, the per-warp shared-memory layouts of the
walk and of the re-rank, and the recently-seen table's tag width.  The header's
functions are plain inline host/device code, so tests/cpp/fast_layout_check.cpp
includes it directly and runs without a GPU."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_walk_and_rerank_layouts(tmp_path):
    exe = str(tmp_path / "fast_layout_check")
    src = os.path.join(ROOT, "tests", "cpp", "fast_layout_check.cpp")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "pickle_b200", "csrc"), "-I" + cuda_inc, src, "-o", exe], check=True)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout + p.stderr
