"""Run the reference binary on a B200 for every golden case.

The binary is oracle/_ref/cuQC_ref, compiled from the reference's main.cu for
sm_100a by oracle/Makefile (built where the reference sources exist and
shipped prebuilt).  For each case it writes, under OUT (default
refbin_out/ at the repository root):
  <name>.refbin.result  the binary's result file
  <name>.refbin.temp    its temp.txt (every emitted set, maximal or not)
  <name>.refbin.log     its stdout (LOADING / ENUMERATION / ... lines)
Cases whose result is empty are skipped: the reference dereferences an empty
prefix tree in RemoveNonMax (main.cu:4834).  Scheduling toggle 1 (static) is
used; it changes the order of work, not the emitted sets.

Usage (GPU box, repository root):  python tests/golden/run_refbin.py [OUT]
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import golden_cases, load_case  # noqa: E402
from oracle import oracle  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "cuQC_ref")


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "refbin_out")
    os.makedirs(out, exist_ok=True)
    summary = {}
    for case in golden_cases():
        name = case["name"]
        g, path, gamma, ms, _ = load_case(case)
        sets, _ = oracle.solve(g, float(gamma), ms, "binary")
        if not sets:
            summary[name] = "skipped: empty result crashes the reference (main.cu:4834)"
            continue
        d = tempfile.mkdtemp(prefix="refbin_")
        res = os.path.join(d, "out.txt")
        p = subprocess.run([BIN, path, gamma, str(ms), res, "1"], cwd=d, capture_output=True,
                           text=True, timeout=600)
        with open(os.path.join(out, name + ".refbin.log"), "w") as f:
            f.write(p.stdout + p.stderr)
        if p.returncode != 0 or not os.path.exists(res):
            summary[name] = "failed rc=%d" % p.returncode
            continue
        shutil.copy(res, os.path.join(out, name + ".refbin.result"))
        shutil.copy(os.path.join(d, "temp.txt"), os.path.join(out, name + ".refbin.temp"))
        summary[name] = "ok"
        print(name, "ok", flush=True)
    with open(os.path.join(out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main()
