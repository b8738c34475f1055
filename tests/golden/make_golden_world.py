"""Writes tests/golden/world_scan.json: the reference's complete hit list for hunt.py's per-seed
workload, from the reference's own CPU scanner (oracle/_ref/lysh, compiled from the reference's
sources by `make -C oracle ref`).

The workload is one world seed over every swamp-hut region of the +-30M world, as hunt.py's CPU
mode scans it (hunt.py:72 WORLD, hunt.py:1390-1392 the `lysh scan` command line): seed
1473884015873122059 (hunt.py:86 SCAN_REFERENCE), regions [-58594, 58594) in x and z, phase-1
floor -50, phase-2 ceiling -50, version 1.19.x~26.1, hits listed.  lysh's phase 1 and phase 2 are
exact, so the list is every hut of that seed whose footprint floor is at or below -50.

    python tests/golden/make_golden_world.py        # about 20 minutes on 8 host cores
    python tests/golden/make_golden_world.py --from-output FILE   # parse a saved run of the same command
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import time

HERE = os.path.dirname(os.path.abspath(__file__))
LYSH = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "lysh")
SEED = 1473884015873122059
RECT = (-58594, 58594, -58594, 58594)
MAX_Y = -50
VERSION = "1.19.x~26.1"


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--from-output", metavar="FILE", help="stdout of the same lysh command, saved earlier")
    args = ap.parse_args()
    threads = os.cpu_count() or 1
    cmd = [LYSH, "scan", "--seed", str(SEED), "--rx0", str(RECT[0]), "--rx1", str(RECT[1]), "--rz0", str(RECT[2]),
           "--rz1", str(RECT[3]), "--threads", str(threads), "--max-y", str(MAX_Y), "--phase2-max-y", str(MAX_Y),
           "--version", VERSION, "--list", "--no-stats"]
    t0 = time.perf_counter()
    if args.from_output:
        with open(args.from_output) as f:
            out = f.read()
        secs = None
    else:
        out = subprocess.run(cmd, capture_output=True, text=True, check=True).stdout
        secs = round(time.perf_counter() - t0, 1)
    hits = []
    for line in out.splitlines():
        t = line.split()
        if line.startswith("hit ") and len(t) >= 6:   # hit rx rz hutX y hutZ ... (lysh main.c printf)
            hits.append({"rx": int(t[1]), "rz": int(t[2]), "hut_x": int(t[3]), "y": int(t[4]), "hut_z": int(t[5])})
    hits.sort(key=lambda h: (h["rz"], h["rx"]))
    # "evaluated": the regions that passed lysh's phase 1 and went through its phase 2
    phase1 = [int(line.split()[-1]) for line in out.splitlines() if line.strip().startswith("evaluated")]
    doc = {"seed": SEED, "rect": list(RECT), "max_y": MAX_Y, "version": VERSION, "hits": hits,
           "phase1_survivors": phase1[0] if phase1 else None,
           "command": "oracle/_ref/lysh " + " ".join(cmd[1:]), "threads": threads, "seconds": secs}
    with open(os.path.join(HERE, "world_scan.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")
    print(f"{len(hits)} hits", f"in {secs} s" if secs else "")


if __name__ == "__main__":
    main()
