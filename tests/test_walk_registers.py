"""The fast walk's result list must live in registers.

RegList keeps 2*S words per lane (keys and ids) in registers, indexed only by
compile-time slot numbers.  A branch on (slot == run-time value) inside an
unrolled loop can be folded by the compiler into one access at a run-time
index, which moves the whole list to local memory: ptxas then reports a
stack frame of 8*S + 8 bytes for the walk kernel, every compare and shift of
the list becomes an L1 load or store, and the c4 mixed batch ran 7-10% slower
with identical results.  This test reads ptxas's report that the build keeps
beside each object (pickle_b200/build.py) and checks that no walk
instantiation has a stack frame that large.  Small spills of a few words are
allowed.
"""
import os
import re

import pytest

from pickle_b200 import build as pk_build

REPORT = os.path.join(pk_build.OBJ, "pk_fast.cu.o.ptxas.txt")


def _walk_frames(text):
    """{(format, slots, parents): stack frame bytes} for every walk_kernel."""
    frames, cur = {}, None
    for line in text.splitlines():
        m = re.search(r"Compiling entry function '(\S+)'", line)
        if m:
            cur = re.search(r"walk_kernelILi(\d+)ELi(\d+)ELi(\d+)E", m.group(1))
            continue
        m = re.search(r"(\d+) bytes stack frame", line)
        if cur and m:
            frames[tuple(int(g) for g in cur.groups())] = int(m.group(1))
            cur = None
    return frames


def test_walk_list_is_not_in_local_memory():
    if not os.path.exists(REPORT):
        pytest.skip("no ptxas report: the library was built before the build kept one")
    with open(REPORT) as f:
        frames = _walk_frames(f.read())
    # two formats x ten list widths x two parent counts
    assert len(frames) == 40, sorted(frames)
    for (trav, slots, parents), frame in frames.items():
        assert frame < 8 * slots + 8, (
            f"walk_kernel<{trav}, {slots}, {parents}> has a {frame}-byte stack frame: its list of "
            f"{2 * slots} words per lane is in local memory")


def test_report_parser_flags_a_list_in_local_memory():
    text = ("ptxas info    : Compiling entry function '_ZN2pk4walk_kernelILi1ELi16ELi1EEEvv' for 'sm_100a'\n"
            "ptxas info    : Function properties for _ZN2pk4walk_kernelILi1ELi16ELi1EEEvv\n"
            "    136 bytes stack frame, 0 bytes spill stores, 0 bytes spill loads\n")
    assert _walk_frames(text) == {(1, 16, 1): 136}
    assert not 136 < 8 * 16 + 8
