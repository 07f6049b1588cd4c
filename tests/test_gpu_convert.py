"""qc_convert's adjacency-list forms, whose two-hop lists are built on the GPU,
against the reference's adjToSer (adjToSer.cpp:45-204) run on the same lists
(fixtures made by tests/golden/make_convert_golden.py): byte-identical
serialized files, including the reference's reading of a final line break as
one more vertex, repeated neighbours, one-way rows and a self loop."""
import os
import subprocess
import tempfile

import pytest

import cuqc_b200 as Q

pytestmark = pytest.mark.gpu

CONV = os.path.join(os.path.dirname(__file__), "golden", "convert")
LISTS = [f for f in sorted(os.listdir(CONV)) if f.endswith((".adj0", ".adj1", ".adj1.rm"))]


def conv(*args):
    return subprocess.run([Q.CONVERT_PATH] + [str(a) for a in args], capture_output=True)


def read(p):
    with open(p, "rb") as f:
        return f.read()


@pytest.mark.parametrize("name", LISTS)
def test_adj2ser_matches_adjToSer(name):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "g.ser")
        p = conv("adj2ser", os.path.join(CONV, name), out)
        assert p.returncode == 0, p.stderr
        assert read(out) == read(os.path.join(CONV, name + ".ser"))


@pytest.mark.parametrize("twohop", [0, 1])
def test_adj2bin_then_bin2ser(twohop):
    # a simple symmetric graph (the binary reader checks that form)
    src = os.path.join(CONV, "edges_c.adj1")
    with tempfile.TemporaryDirectory() as d:
        b = os.path.join(d, "g.bin")
        s = os.path.join(d, "g.ser")
        assert conv("adj2bin", src, b, twohop).returncode == 0
        p = conv("bin2ser", b, s)
        assert p.returncode == 0, p.stderr
        assert read(s) == read(src + ".ser")


def test_adj2ser_rejects_ids_beyond_the_list():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "a.adj")
        with open(src, "w") as f:
            f.write("1\n0 7")
        p = conv("adj2ser", src, os.path.join(d, "o.ser"))
        assert p.returncode != 0 and b"beyond" in p.stderr


def test_mine_files_streams_result_files():
    # graph files mined one after another, each result written on a host
    # thread while the next graph is mined: every file equals the reference
    # CPU path's result file for that graph
    import json
    from conftest import GOLDEN, golden_cases

    cases = [c for c in golden_cases() if c.get("stored_graph")][:6]
    with tempfile.TemporaryDirectory() as d, Q.Context(device=0) as ctx:
        jobs = [(os.path.join(GOLDEN, c["name"] + ".graph"), float(c["gamma"]), int(c["min_size"]),
                 os.path.join(d, c["name"] + ".txt")) for c in cases]
        stats = ctx.mine_files(jobs)
        assert len(stats) == len(cases)
        for c, job in zip(cases, jobs):
            assert read(job[3]) == read(os.path.join(GOLDEN, c["name"] + ".refcpu.result"))
