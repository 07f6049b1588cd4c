"""The graph-format tools (qc_convert, cuqc_b200/csrc/convert.cpp) against the
reference's own converters' outputs: edgeToAdj.py (Mike12041204/cuQC
edgeToAdj.py:5-50) and rmEmptyVert.py (rmEmptyVert.py:29-63), fixtures made by
tests/golden/make_convert_golden.py.  The adjToSer form, whose two-hop lists
are built on the GPU, is in test_gpu_convert.py."""
import os
import subprocess
import tempfile

import pytest

import cuqc_b200 as Q

CONV = os.path.join(os.path.dirname(__file__), "golden", "convert")
CASES = ("edges_a", "edges_b", "edges_c")


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(Q.CONVERT_PATH):
        Q.build()


def conv(*args):
    return subprocess.run([Q.CONVERT_PATH] + [str(a) for a in args], capture_output=True)


def read(p):
    with open(p, "rb") as f:
        return f.read()


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("dup", [0, 1])
def test_edges2adj_matches_edgeToAdj(case, dup):
    p = conv("edges2adj", os.path.join(CONV, case + ".txt"), dup)
    assert p.returncode == 0, p.stderr
    assert p.stdout == read(os.path.join(CONV, "%s.adj%d" % (case, dup)))
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "a.adj")
        assert conv("edges2adj", os.path.join(CONV, case + ".txt"), dup, out).returncode == 0
        assert read(out) == p.stdout


@pytest.mark.parametrize("case", CASES)
def test_rmempty_matches_rmEmptyVert(case):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "r.adj")
        p = conv("rmempty", os.path.join(CONV, case + ".adj1"), out)
        assert p.returncode == 0, p.stderr
        assert read(out) == read(os.path.join(CONV, case + ".adj1.rm"))


def test_rmempty_rejects_a_name_without_a_line():
    # one-way lists can name a vertex whose line is empty (rmEmptyVert.py
    # raises KeyError there)
    with tempfile.TemporaryDirectory() as d:
        p = conv("rmempty", os.path.join(CONV, "edges_a.adj0"), os.path.join(d, "r.adj"))
        assert p.returncode != 0 and b"no neighbours" in p.stderr


def test_edges2adj_rejects_malformed_lines():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "e.txt")
        with open(src, "w") as f:
            f.write("1 2\n3\n")
        p = conv("edges2adj", src, 1)
        assert p.returncode != 0 and b"line 2" in p.stderr


def test_edges2adj_crlf_and_no_final_newline():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "e.txt")
        with open(src, "wb") as f:
            f.write(b"0 2\r\n2 1\r\n1 3")
        p = conv("edges2adj", src, 1)
        assert p.returncode == 0
        assert p.stdout == b"2\n2 3\n0 1\n1\n"


@pytest.mark.parametrize("name", ["small00", "small03", "small09"])
def test_serialized_binary_round_trip(name):
    src = os.path.join(os.path.dirname(__file__), "golden", name + ".graph")
    if not os.path.exists(src):
        pytest.skip("graph not stored")
    with tempfile.TemporaryDirectory() as d:
        b = os.path.join(d, "g.bin")
        s = os.path.join(d, "g.ser")
        assert conv("ser2bin", src, b).returncode == 0
        assert read(b)[:8] == b"QCSRBIN1"
        assert conv("bin2ser", b, s).returncode == 0
        assert read(s) == read(src)


def test_usage():
    p = conv("nonsense")
    assert p.returncode == 1 and b"Usage: qc_convert" in p.stderr
