"""Generate tests/golden/cfg3_batch.json: the batched workload's instances.

The batched configuration draws independent instances (cuqc_b200.graphs.
batch_instance: n log-uniform 200-5000, Chung-Lu exponent 2.1 with mean
degree 10-50, 1-20 planted groups of size 10-40 at density 0.8-1.0, gamma in
{0.6, 0.7, 0.8, 0.9, 0.95}, min_size 5-30).  Many draws have search trees of
hundreds of millions of tasks or more (dense cores at gamma 0.6-0.8 with small
min_size), which no single run finishes in minutes.  The workload therefore
keeps the first 256 draws (in index order) whose search tree, expanded by the
CPU oracle, stays within a fixed budget of tasks and of parent-task vertices
read by branches; the budget, the kept indices and every kept instance's
maximal-set count and result digest are recorded so the GPU runs can be
checked against the oracle.

Run from the repository root:  python tests/golden/make_batch_manifest.py
"""
import hashlib
import json
import multiprocessing as mp
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

MAX_TASKS = 200_000
MAX_PARENT_VERTICES = 20_000_000
WANT = 256
OUT = os.path.join(ROOT, "tests", "golden", "cfg3_batch.json")


def result_digest(sets):
    text = "".join("%d %s \n" % (len(s), " ".join(map(str, s))) for s in sets)
    return hashlib.sha1(text.encode()).hexdigest()


def screen(i):
    from cuqc_b200 import graphs
    from oracle import oracle
    g, gamma, ms = graphs.batch_instance(i)
    try:
        sets, st = oracle.solve(g, float(gamma), ms, max_tasks=MAX_TASKS,
                                max_parent_vertices=MAX_PARENT_VERTICES)
    except oracle.BudgetExceeded:
        return {"i": i, "kept": False}
    return {"i": i, "kept": True, "n": g.n, "gamma": gamma, "min_size": ms,
            "tasks": st["tasks"], "maximal": len(sets), "digest": result_digest(sets)}


def main():
    ctx = mp.get_context("spawn")
    kept, screened, start = [], 0, 0
    with ctx.Pool(os.cpu_count() or 1) as pool:
        while len(kept) < WANT:
            chunk = list(range(start, start + 64))
            start += 64
            for r in pool.map(screen, chunk):
                screened += 1
                if r["kept"] and len(kept) < WANT:
                    kept.append(r)
            print("screened %d, kept %d" % (screened, len(kept)), flush=True)
    kept.sort(key=lambda r: r["i"])
    last = kept[-1]["i"]
    doc = {"generator": "cuqc_b200.graphs.batch_instance",
           "budget": {"max_tasks": MAX_TASKS, "max_parent_vertices": MAX_PARENT_VERTICES},
           "screened_through_index": last, "kept": len(kept),
           "kept_fraction": len(kept) / (last + 1),
           "instances": [{k: r[k] for k in ("i", "n", "gamma", "min_size", "tasks", "maximal",
                                            "digest")} for r in kept]}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=0)
    print("wrote", OUT, "kept", len(kept), "of", last + 1)


if __name__ == "__main__":
    main()
