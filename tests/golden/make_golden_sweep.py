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

Second step, on any machine with g++ (no GPU):

    python tests/golden/make_golden_sweep.py --cpu <reference root>

adds the same per-seed start counts from the reference's room walk header compiled on the CPU
(sweep_world_counts.cpp), once with plain -O2 and once with -O2 -fwrapv, and the starts whose
region re-draws nextInt(24) under each build.  The header's re-draw test (room_core.h:94, :100) is
signed 32-bit arithmetic that overflows exactly when a re-draw is due: the optimised builds drop
the loop (the -O2 counts equal the GPU engine's), while with defined wrapping the loop runs as
java.util.Random.nextInt and lysh's lysh_lcg_next_int_bound (rng.c:213-226) do.
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


def cpu_counts(ref_root: str, s48s: list[int], wrap: bool) -> tuple[list[int], list[tuple[int, ...]]]:
    """Whole-world start counts of the reference's room walk (sweep_world_counts.cpp compiled against
    its engine/gpu/room_core.h), with plain -O2 or with -O2 -fwrapv; and the starts whose region
    re-draws nextInt(24), as (s48, rx, rz, chunk x, chunk z)."""
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sweep_world_counts.cpp")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "counts")
        flags = ["-O2", "-fopenmp"] + (["-fwrapv"] if wrap else [])
        subprocess.run(["g++", *flags, "-I", os.path.join(ref_root, "engine", "gpu"), src, "-o", exe], check=True)
        r = subprocess.run([exe, *map(str, s48s)], capture_output=True, text=True, check=True, timeout=3600)
    starts, redraw = [], []
    for line in r.stdout.splitlines():
        p = line.split()
        if p[0] == "seed":
            starts.append(int(p[3]))
        elif p[0] == "redraw_start":
            redraw.append(tuple(int(x) for x in p[1:]))
    return starts, sorted(redraw)


def add_cpu_counts(path: str, ref_root: str) -> None:
    """Adds the CPU counts of both builds to an existing fixture."""
    g = dict(np.load(path))
    s48s = [int(s) for s in g["s48"]]
    for wrap, tag in ((False, "o2"), (True, "wrapv")):
        starts, redraw = cpu_counts(ref_root, s48s, wrap)
        g[f"cpu_starts_{tag}"] = np.array(starts, np.uint64)
        g[f"redraw_starts_{tag}"] = np.array(redraw, np.int64).reshape(-1, 5)
        print(f"{tag}: starts {starts}, re-draw starts {redraw}")
    np.savez(path, **g)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "deep_sweep.npz"))
    ap.add_argument("--cpu", metavar="REF_ROOT",
                    help="instead of running the reference's GPU engine, add to the fixture at --out the "
                         "whole-world counts of the reference's room walk built on the CPU with -O2 and with "
                         "-O2 -fwrapv (REF_ROOT: the reference's root)")
    args = ap.parse_args()
    if args.cpu:
        add_cpu_counts(args.out, args.cpu)
        return
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
