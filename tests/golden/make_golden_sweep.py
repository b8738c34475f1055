"""Writes the Deep Dive forward sweep's golden counts from the reference's own GPU engine.

Needs a GPU and the reference engine built here first (`make -C oracle refsolver REF=<reference root>`,
which compiles engine/gpu/hut_lookup_v4_source.cu into oracle/_ref/hut_lookup_v4).  On the GPU machine:

    python tests/golden/make_golden_sweep.py --out deep_sweep.npz

then copy the file to tests/golden/deep_sweep.npz.

The reference's forward mode (`hut_lookup_v4 --catalog C --first-index F --count N --max-height -54`,
engine/gpu/hut_lookup_v4_source.cu:1504-1530) walks every hut region of the +-30M world for each
structure seed s48 = (index * 0x9E3779B97F4A7D + 0x2545F4914F6CDD) mod 2^48 (:27-29, :1505), counts
the mineshaft starts under huts and probes each start's carver state in the layout catalogue
(sweepProbeKernel, :77-99), and prints "S48 s (index i): A hut starts, B catalogue matches, C terrain
survivors" per structure seed.  A random catalogue matches nothing (one start in 2^48 would), so
the catalogue here is planted: the carver states of two starts of each structure seed near the
origin (from the C restatement oracle/witch_oracle.c, wo_deep_starts) plus three decoy layouts.
The fixture keeps the structure seeds, the catalogue, and the reference's start and match counts
per structure seed (its terrain survivors too, for the record: its terrain gates are its own staged
tests, not lysh's phase 1).
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
REF_ENGINE = os.path.join(ROOT, "oracle", "_ref", "hut_lookup_v4")

FIRST, COUNT = 1000, 3
MASK48 = (1 << 48) - 1


def forward_s48(index: int) -> int:
    """The reference forward mode's structure seed of an index."""
    return (index * 0x9E3779B97F4A7D + 0x2545F4914F6CDD) & MASK48


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "deep_sweep.npz"))
    args = ap.parse_args()
    import bind
    port = bind.Port()
    s48s = [forward_s48(FIRST + i) for i in range(COUNT)]
    layouts, values = [], []
    for s in s48s:
        rows = port.deep_starts([s], (-40, 40, -40, 40))
        for r in (rows[0], rows[-1]):
            layouts.append(int(r[5]) & MASK48)
            values.append(300 + len(values) | (200 + len(values)) << 10)
    rng = np.random.default_rng(11)
    for _ in range(3):
        layouts.append(int(rng.integers(0, 1 << 48)))
        values.append(1 | 1 << 10)
    with tempfile.TemporaryDirectory() as tmp:
        cat = os.path.join(tmp, "catalog.txt")
        with open(cat, "w") as f:
            for x, v in zip(layouts, values):
                f.write(f"{x} {v & 0x3FF} {v >> 10}\n")
        out = os.path.join(tmp, "ref.csv")
        cmd = [REF_ENGINE, "--catalog", cat, "--first-index", str(FIRST), "--count", str(COUNT), "--max-height", "-54",
               "--out", out]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            raise SystemExit(f"reference engine failed ({r.returncode}): {r.stderr[-2000:]}")
        starts, matches, surv = [], [], []
        for line in r.stderr.splitlines():
            m = re.match(r"S48 (-?\d+) \(index (\d+)\): (\d+) hut starts, (\d+) catalogue matches, (\d+) terrain", line)
            if m:
                assert int(m.group(1)) == s48s[int(m.group(2)) - FIRST], line
                starts.append(int(m.group(3)))
                matches.append(int(m.group(4)))
                surv.append(int(m.group(5)))
        print(r.stdout.strip(), file=sys.stderr)
        print("\n".join(l for l in r.stderr.splitlines() if l.startswith("S48")), file=sys.stderr)
        rows = []
        with open(out) as f:
            next(f, None)
            for line in f:
                p = line.strip().split(",")
                if len(p) >= 4:
                    rows.append((int(p[0]), int(p[1]), int(p[2]), int(p[3])))
    if len(starts) != COUNT:
        raise SystemExit("the reference printed no per-seed lines")
    np.savez(args.out, s48=np.array(s48s, np.int64), layouts=np.array(layouts, np.uint64),
             values=np.array(values, np.uint32), ref_starts=np.array(starts, np.uint64),
             ref_matches=np.array(matches, np.uint64), ref_terrain_survivors=np.array(surv, np.uint64),
             ref_survivor_rows=np.array(rows, np.int64).reshape(-1, 4))
    print(f"wrote {args.out}: starts {starts}, matches {matches}, terrain survivors {surv}")


if __name__ == "__main__":
    main()
