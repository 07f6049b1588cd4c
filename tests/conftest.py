import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "emu"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def load_case(case):
    """(graph, path, gamma string, min_size, reference CPU-path result text)"""
    from cuqc_b200 import graphs
    import hashlib
    import tempfile

    if case["stored_graph"]:
        path = os.path.join(GOLDEN, case["name"] + ".graph")
        g = graphs.read_serialized(path)
    else:
        g = getattr(graphs, case["generator"])(**case["kwargs"])
        path = os.path.join(tempfile.mkdtemp(), case["name"] + ".graph")
        graphs.write_serialized(g, path)
    with open(path, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == case["graph_sha256"], \
            "generator output drifted for " + case["name"]
    with open(os.path.join(GOLDEN, case["name"] + ".refcpu.result")) as f:
        expected = f.read()
    return g, path, case["gamma"], case["min_size"], expected


def parse_result(text):
    return [tuple(int(x) for x in line.split()[1:]) for line in text.splitlines()]


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
