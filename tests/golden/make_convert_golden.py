"""Builds the fixtures of the graph-format tools (tests/golden/convert/) by
running the reference's own converters on small seeded inputs: edgeToAdj.py
and rmEmptyVert.py with this interpreter, and adjToSer.cpp as compiled by
oracle/Makefile (oracle/_ref/adjToSer).  Run where the reference sources are
(QC_REFERENCE_DIR, default /root/reference); the outputs are committed.

    python tests/golden/make_convert_golden.py
"""
import os
import random
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "convert")
REF = os.environ.get("QC_REFERENCE_DIR", "/root/reference")
ADJTOSER = os.path.join(HERE, "..", "..", "oracle", "_ref", "adjToSer")


def edge_inputs():
    rng = random.Random(20261204)
    cases = {}
    # a random graph on 0..24 with some repeated and reversed edges
    e = [(rng.randrange(25), rng.randrange(25)) for _ in range(60)]
    e = [(u, v) for u, v in e if u != v]
    e += [(v, u) for u, v in e[:6]] + e[6:9]
    cases["edges_a"] = e
    # ids with gaps (vertices without edges) and a self loop
    cases["edges_b"] = [(2, 5), (5, 9), (9, 2), (12, 5), (7, 7), (12, 9), (15, 2)]
    # a path written one way only
    cases["edges_c"] = [(i, i + 1) for i in range(10)]
    return cases


def run(cmd, stdout=None):
    subprocess.check_call(cmd, stdout=stdout)


def main():
    os.makedirs(OUT, exist_ok=True)
    for name, edges in edge_inputs().items():
        src = os.path.join(OUT, name + ".txt")
        with open(src, "w") as f:
            f.write("".join("%d %d\n" % (u, v) for u, v in edges))
        for dup in (0, 1):
            adj = os.path.join(OUT, "%s.adj%d" % (name, dup))
            with open(adj, "w") as f:
                run([sys.executable, os.path.join(REF, "edgeToAdj.py"), src, str(dup)], stdout=f)
            run([ADJTOSER, adj, adj + ".ser"])
            if dup == 1:
                # the reference pipeline: drop empty vertices, then serialize
                # (one-way lists can name a vertex without a line of its own,
                # which rmEmptyVert.py rejects)
                rm = os.path.join(OUT, "%s.adj%d.rm" % (name, dup))
                run([sys.executable, os.path.join(REF, "rmEmptyVert.py"), adj, rm])
                run([ADJTOSER, rm, rm + ".ser"])
    print("fixtures in", OUT)


if __name__ == "__main__":
    main()
