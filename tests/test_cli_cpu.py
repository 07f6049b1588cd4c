"""The drop-in CLI's argument checks (before any device use), as the
reference's main (main.cu:427-453)."""
import os
import tempfile

import pytest

import cuqc_b200 as Q
from cuqc_b200 import graphs


@pytest.fixture(scope="module")
def gfile():
    if not os.path.exists(Q.CLI_PATH):
        Q.build()
    d = tempfile.mkdtemp()
    p = os.path.join(d, "g.txt")
    graphs.write_serialized(graphs.random_small(20, 0.3, 1), p)
    return p


def run(args):
    import subprocess
    p = subprocess.run([Q.CLI_PATH] + args, capture_output=True, text=True)
    return p.returncode, p.stdout


def test_usage(gfile):
    rc, out = run([gfile])
    assert rc == 1 and out.startswith("Usage: ./main <graph_file> <gamma> <min_size>")


def test_invalid_graph_file():
    rc, out = run(["/nonexistent", "0.9", "5", "/tmp/o.txt", "0"])
    assert rc == 1 and out.strip() == "invalid graph file"


@pytest.mark.parametrize("gamma", ["0.49", "1.01", "abc"])
def test_gamma_range(gfile, gamma):
    rc, out = run([gfile, gamma, "5", "/tmp/o.txt", "0"])
    assert rc == 1 and "minimum degree ratio must be between .5 and 1 inclusive" in out


@pytest.mark.parametrize("ms", ["1", "0", "-3"])
def test_min_size(gfile, ms):
    rc, out = run([gfile, "0.9", ms, "/tmp/o.txt", "0"])
    assert rc == 1 and "minimum size must be greater than 1" in out


def test_bad_sched_is_reported_and_run_continues(gfile, has_gpu):
    rc, out = run([gfile, "0.9", "5", os.path.join(tempfile.mkdtemp(), "o.txt"), "7"])
    assert "scheduling toggle must be 0 or 1" in out
    assert ">:PRE-PROCESSING" in out  # continued past the check
    if not has_gpu:
        assert rc != 0 and "no CUDA device" in out
