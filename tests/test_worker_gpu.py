"""GPU: the phase1_scan worker protocol as hunt.py drives it (GpuScanWorker, hunt.py:1276-1332):
===WORKER_READY===, one request per stdin line, CSV out, ===SCAN_DONE rc=0===, a bad line
answered with ===SCAN_ERROR...=== without stopping the worker, clean exit on EOF."""
from __future__ import annotations

import csv
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def read_csv(path):
    with open(path) as f:
        rows = list(csv.reader(f))
    assert rows[0] == ["seed", "chunkX", "chunkZ", "blockX", "blockZ", "gpuEst"]
    return [(int(r[0]), int(r[1]), int(r[2]), int(r[3]), int(r[4])) for r in rows[1:]]


def test_worker_protocol(wg, engine, tmp_path):
    seed = 1473884015873122059
    p = subprocess.Popen([wg.WORKER_PATH, "--worker"], stdin=subprocess.PIPE, stdout=subprocess.PIPE,
                         stderr=subprocess.PIPE, text=True, bufsize=1, cwd=tmp_path)
    try:
        assert p.stdout.readline().strip() == "===WORKER_READY==="

        def ask(line):
            p.stdin.write(line + "\n")
            p.stdin.flush()
            while True:
                out = p.stdout.readline()
                assert out, "worker died"
                if out.startswith("===SCAN_DONE") or out.startswith("===SCAN_ERROR"):
                    return out.strip()

        # hunt.py's request for a 40,000-block area (ScanRun.rect: r = 40000 // 512 + 1)
        assert ask(f"--seed {seed} --min-region-x -79 --max-region-x 79 --min-region-z -79 "
                   f"--max-region-z 79 --max-height -50 --out cands.csv") == "===SCAN_DONE rc=0==="
        rows = read_csv(tmp_path / "cands.csv")
        assert rows == [(seed, -987, -1073, -15792, -17168)]
        assert ask("--seed 1 --bogus-flag") == "===SCAN_ERROR: bad request line==="
        # a UTF-8 BOM is stripped, negative seeds wrap like strtoull, seed lists work
        (tmp_path / "seeds.txt").write_text(f"{seed}, -5\n 17\n")
        assert ask("\ufeff--seed-list seeds.txt --min-region-x -79 --max-region-x 79 --min-region-z -79 "
                   "--max-region-z 79 --max-height -54 --out b.csv") == "===SCAN_DONE rc=0==="
        got = read_csv(tmp_path / "b.csv")
        want = engine.seed_check(seeds=[seed, -5, 17], rect=(-79, 79, -79, 79), max_height=-50).candidates
        assert got == [(int(c["seed"]), int(c["chunk_x"]), int(c["chunk_z"]), int(c["chunk_x"]) * 16,
                        int(c["chunk_z"]) * 16) for c in want]
        assert ask("--seed-gen 2 65536 --min-region-x -4 --max-region-x 5 --min-region-z -4 --max-region-z 5 "
                   "--max-height -50 --out g.csv") == "===SCAN_DONE rc=0==="
        assert read_csv(tmp_path / "g.csv") == []
    finally:
        p.stdin.close()
        rc = p.wait(timeout=60)
    assert rc == 0


def test_single_shot_cli(wg, engine, tmp_path):
    r = subprocess.run([wg.WORKER_PATH, "--seed-gen", "2", "4194304", "--min-region-x", "-4", "--max-region-x", "5",
                        "--min-region-z", "-4", "--max-region-z", "5", "--max-height", "-50", "--out", "c.csv"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "candidates=52" in r.stdout
    rows = read_csv(tmp_path / "c.csv")
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c2_4m_survivors.npz"))["survivors"]
    assert rows == [(int(c["seed"]), int(c["chunk_x"]), int(c["chunk_z"]), int(c["chunk_x"]) * 16,
                     int(c["chunk_z"]) * 16) for c in g]
