"""Writes the Deep Dive solver's golden hits from the reference's own GPU engine.

Needs a GPU and the reference solver built here first (`make -C oracle refsolver REF=<reference root>`, which compiles
engine/gpu/hut_lookup_v4_source.cu into oracle/_ref/hut_lookup_v4).  On the GPU machine:

    python tests/golden/make_golden_solve.py --out deep_solve.npz

then copy the file to tests/golden/deep_solve.npz.  Each case runs the reference as hunt.py does
(`hut_lookup_v4 --catalog C --solve-only --solve5 --plan P --first-index F --count N --dump-hits H`,
hunt.py:947-952) on a one-line plan and records every hit (structure seed, chunk x, chunk z).
The layouts are the three catalogued ones of data/hunt/58 and data/hunt/59 (layout_catalog.txt),
with the regime and offset class each case names.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_SOLVER = os.path.join(ROOT, "oracle", "_ref", "hut_lookup_v4")

# (layout, air hi, air lo) of the reference's layout catalogues
LAYOUTS = {231564844655014: (331, 331), 156186219368766: (321, 303), 270840896143627: (322, 316)}
# (layout, regime "XZ", class, first group, groups)
CASES = [(231564844655014, "22", "odd", 0, 2),
         (231564844655014, "00", "odd", 5, 2),
         (156186219368766, "21", "odd", 777, 1),
         (270840896143627, "00", "u2", 0, 1),
         (156186219368766, "00", "eq", 3, 1)]


def run_case(tmp: str, layout: int, regime: str, cls: str, first: int, count: int) -> np.ndarray:
    cat = os.path.join(tmp, "catalog.txt")
    plan = os.path.join(tmp, "plan.txt")
    hits = os.path.join(tmp, "hits.csv")
    with open(cat, "w") as f:
        hi, lo = LAYOUTS[layout]
        f.write(f"{layout} {hi} {lo}\n")
    with open(plan, "w") as f:
        f.write(f"{layout} {regime} {cls}\n")
    if os.path.exists(hits):
        os.remove(hits)
    cmd = [REF_SOLVER, "--catalog", cat, "--solve-only", "--solve5", "--plan", plan, "--first-index", str(first),
           "--count", str(count), "--quiet", "--dump-hits", hits, "--out", os.path.join(tmp, "dummy.csv")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    print(r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "", flush=True)
    if r.returncode != 0:
        raise SystemExit(f"reference solver failed ({r.returncode}): {r.stderr[-2000:]}")
    rows = []
    with open(hits) as f:
        for line in f:
            p = line.strip().split(",")
            if len(p) >= 4:
                rows.append((int(p[0]), int(p[1]), int(p[2]), int(p[3])))
    rows.sort()
    return np.array(rows, dtype=np.int64).reshape(-1, 4)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "deep_solve.npz"))
    args = ap.parse_args()
    arrays = {"cases": np.array([(lay, int(rg[0]), int(rg[1]), {"odd": 1, "u2": 2, "eq": 3}[cls], first, n)
                                 for lay, rg, cls, first, n in CASES], dtype=np.int64)}
    with tempfile.TemporaryDirectory() as tmp:
        for k, (lay, rg, cls, first, n) in enumerate(CASES):
            hits = run_case(tmp, lay, rg, cls, first, n)
            print(f"case {k}: layout {lay} regime {rg} {cls} groups {first}..{first + n}: {len(hits)} hits", flush=True)
            arrays[f"hits{k}"] = hits
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez_compressed(args.out, **arrays)


if __name__ == "__main__":
    main()
