"""Generate the golden fixtures in this directory.

Each case is a seeded synthetic graph (cuqc_b200.graphs) in the reference's
serialized format plus result files the REFERENCE produced for it:
  <name>.refcpu.result  the reference cuQC's own serial CPU path (its
                        initialize_tasks, h_expand_level and RemoveNonMax,
                        compiled from the reference sources by oracle/Makefile
                        into oracle/_ref/libqc_refcpu.so), made by this script;
  <name>.refbin.result  the reference binary (built from main.cu for sm_100a)
                        run once on a B200; these and its temp.txt files
                        (*.refbin.temp) and logs (refbin_logs/) are frozen
                        records -- the binary is not built or run again
                        (it faulted on small inputs).  Large graphs are not stored: their generator
parameters and a digest of the serialized text are, so the tests regenerate
them and check the digest first.

Run from the repository root (needs the reference sources, i.e. this
container):  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from cuqc_b200 import graphs  # noqa: E402
from oracle import oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, generator, kwargs, gamma string, min_size, store graph?)
CASES = []
for i in range(16):
    rng = np.random.default_rng(1000 + i)
    n = int(rng.integers(12, 48))
    p = float(rng.uniform(0.12, 0.45))
    planted = int(rng.integers(0, 4))
    size = int(rng.integers(5, 12))
    dens = float(rng.uniform(0.85, 1.0))
    gamma = ["0.5", "0.6", "0.7", "0.75", "0.8", "0.85", "0.9", "0.95", "1"][i % 9]
    ms = int(rng.integers(3, 8))
    CASES.append(("small%02d" % i, "random_small",
                  dict(n=n, p=p, seed=1000 + i, planted=planted, size=size, density=dens),
                  gamma, ms, True))
CASES.append(("er1000_planted", "erdos_renyi_planted",
              dict(n=1000, p=0.02, groups=5, group_size=30, density=0.95, seed=1), "0.9", 20, False))
CASES.append(("er300_planted", "erdos_renyi_planted",
              dict(n=300, p=0.03, groups=3, group_size=16, density=0.95, seed=11), "0.8", 10, False))


def make(gen, kw):
    return getattr(graphs, gen)(**kw)


def digest(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def main():
    manifest = []
    tmp = os.path.join(HERE, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    for name, gen, kw, gamma, ms, store in CASES:
        g = make(gen, kw)
        gpath = os.path.join(HERE if store else tmp, name + ".graph")
        graphs.write_serialized(g, gpath)
        text, emitted = oracle.refcpu_run(gpath, gamma, ms, workdir=tmp)
        with open(os.path.join(HERE, name + ".refcpu.result"), "w") as f:
            f.write(text)
        manifest.append(dict(name=name, generator=gen, kwargs=kw, gamma=gamma, min_size=ms,
                             stored_graph=store, graph_sha256=digest(gpath),
                             refcpu_maximal=text.count("\n"), emitted=int(oracle.unpack(emitted).__len__()),
                             ))
        print(name, "maximal", manifest[-1]["refcpu_maximal"], "emitted", manifest[-1]["emitted"], flush=True)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
