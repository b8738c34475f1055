"""GPU: hunt.py's per-seed workload at full size, against the reference's own complete answer.

hunt.py's GPU mode sends the phase1_scan worker one seed over every swamp-hut region of the
+-30M world (hunt.py:72 WORLD, hunt.py:1305 the request line).  tests/golden/world_scan.json
holds the reference CPU scanner's (lysh's) complete hit list for seed 1473884015873122059
(hunt.py:86 SCAN_REFERENCE) over that world at floor -50, made by
tests/golden/make_golden_world.py.  The worker's rows (the exact hit set, floor y in the sixth
column) must be that list, hut for hut and floor for floor: 1.37e10 (seed, region) checks through
phase 1, then phase 2 of every phase-1 survivor, bit-exact end to end.  The phase-1 survivors
through the C ABI (wg_seed_check) must number what lysh evaluated in its phase 2."""
from __future__ import annotations

import csv
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "world_scan.json")


def test_whole_world_worker_equals_reference_hit_list(wg, tmp_path):
    with open(GOLDEN) as f:
        ref = json.load(f)
    r = ref["rect"]
    cmd = [wg.WORKER_PATH, "--seed", str(ref["seed"]), "--min-region-x", str(r[0]), "--max-region-x", str(r[1]),
           "--min-region-z", str(r[2]), "--max-region-z", str(r[3]), "--max-height", str(ref["max_y"]),
           "--out", str(tmp_path / "cands.csv")]
    subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=600)
    with open(tmp_path / "cands.csv") as f:
        rows = list(csv.reader(f))
    assert rows[0] == ["seed", "chunkX", "chunkZ", "blockX", "blockZ", "gpuEst"]
    got = sorted((int(x[3]), int(x[4]), int(x[5])) for x in rows[1:])
    want = sorted((h["hut_x"], h["hut_z"], h["y"]) for h in ref["hits"])
    assert len(want) > 0
    assert got == want
    assert all(int(x[0]) == ref["seed"] for x in rows[1:])
    assert all(int(x[1]) * 16 == int(x[3]) and int(x[2]) * 16 == int(x[4]) for x in rows[1:])


def test_whole_world_phase1_survivors_equal_reference_count(wg, engine):
    with open(GOLDEN) as f:
        ref = json.load(f)
    res = engine.seed_check(seeds=[ref["seed"]], rect=tuple(ref["rect"]), max_height=ref["max_y"],
                            version=ref["version"])
    assert len(res.candidates) == ref["phase1_survivors"]
    got = {(int(c["chunk_x"]) * 16, int(c["chunk_z"]) * 16) for c in res.candidates}
    assert all((h["hut_x"], h["hut_z"]) in got for h in ref["hits"])
