"""GPU: the phase1_scan worker protocol as hunt.py drives it (GpuScanWorker, hunt.py:1276-1332):
===WORKER_READY===, one request per stdin line, CSV out, ===SCAN_DONE rc=0===, a bad line
answered with ===SCAN_ERROR...=== without stopping the worker, clean exit on EOF.

By default the worker writes the exact hit set (phase-1 survivors that lysh_eval_hut accepts at
the phase-2 ceiling), with the hut's floor y in the 6th column; --phase1-candidates writes the
phase-1 survivors instead.  hunt.py reads only the first three columns and re-confirms every row
with `lysh hut` at a ceiling <= -50, so both outputs give it the same results."""
from __future__ import annotations

import csv
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def read_csv(path, floor=False):
    with open(path) as f:
        rows = list(csv.reader(f))
    assert rows[0] == ["seed", "chunkX", "chunkZ", "blockX", "blockZ", "gpuEst"]
    if floor:
        return [(int(r[0]), int(r[1]), int(r[2]), int(r[3]), int(r[4]), int(r[5])) for r in rows[1:]]
    return [(int(r[0]), int(r[1]), int(r[2]), int(r[3]), int(r[4])) for r in rows[1:]]


def exact_rows(engine, cands, max_y):
    """The worker's default output for phase-1 survivors `cands`: the huts lysh_eval_hut accepts."""
    if len(cands) == 0:
        return []
    res = engine.eval_huts(cands["seed"], cands["chunk_x"].astype(np.int64) * 16,
                           cands["chunk_z"].astype(np.int64) * 16, max_y=max_y)
    return [(int(c["seed"]), int(c["chunk_x"]), int(c["chunk_z"]), int(c["chunk_x"]) * 16, int(c["chunk_z"]) * 16,
             int(r["avg_y"])) for c, r in zip(cands, res) if r["ok"]]


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
        # hunt.py SCAN_REFERENCE: /tp -15792 -54 -17168, the floor in the 6th column
        assert read_csv(tmp_path / "cands.csv", floor=True) == [(seed, -987, -1073, -15792, -17168, -54)]
        assert ask("--seed 1 --bogus-flag") == "===SCAN_ERROR: bad request line==="
        # a UTF-8 BOM is stripped, negative seeds wrap like strtoull, seed lists work; the phase-2
        # ceiling is --max-height as given (-54) while phase 1 runs at the clamped -50
        (tmp_path / "seeds.txt").write_text(f"{seed}, -5\n 17\n")
        assert ask("\ufeff--seed-list seeds.txt --min-region-x -79 --max-region-x 79 --min-region-z -79 "
                   "--max-region-z 79 --max-height -54 --out b.csv") == "===SCAN_DONE rc=0==="
        want = engine.seed_check(seeds=[seed, -5, 17], rect=(-79, 79, -79, 79), max_height=-50).candidates
        assert read_csv(tmp_path / "b.csv", floor=True) == exact_rows(engine, want, -54)
        assert ask("\ufeff--seed-list seeds.txt --min-region-x -79 --max-region-x 79 --min-region-z -79 "
                   "--max-region-z 79 --max-height -54 --phase1-candidates --out p.csv") == "===SCAN_DONE rc=0==="
        assert read_csv(tmp_path / "p.csv") == [(int(c["seed"]), int(c["chunk_x"]), int(c["chunk_z"]),
                                                 int(c["chunk_x"]) * 16, int(c["chunk_z"]) * 16) for c in want]
        assert len(want) >= 1
        assert ask("--seed-gen 2 65536 --min-region-x -4 --max-region-x 5 --min-region-z -4 --max-region-z 5 "
                   "--max-height -50 --out g.csv") == "===SCAN_DONE rc=0==="
        assert read_csv(tmp_path / "g.csv") == []
    finally:
        p.stdin.close()
        rc = p.wait(timeout=60)
    assert rc == 0


def test_single_shot_cli(wg, engine, tmp_path):
    args = [wg.WORKER_PATH, "--seed-gen", "2", "4194304", "--min-region-x", "-4", "--max-region-x", "5",
            "--min-region-z", "-4", "--max-region-z", "5", "--max-height", "-50"]
    r = subprocess.run(args + ["--phase1-candidates", "--out", "c.csv"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "candidates=52" in r.stdout
    rows = read_csv(tmp_path / "c.csv")
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "c2_4m_survivors.npz"))["survivors"]
    assert rows == [(int(c["seed"]), int(c["chunk_x"]), int(c["chunk_z"]), int(c["chunk_x"]) * 16,
                     int(c["chunk_z"]) * 16) for c in g]
    # the default output: those 52 through phase 2 at the ceiling -50
    r = subprocess.run(args + ["--out", "h.csv"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "phase 2: 52 phase-1 survivors" in r.stdout
    assert read_csv(tmp_path / "h.csv", floor=True) == exact_rows(engine, g, -50)


def test_exact_hits_follow_the_phase2_ceiling(wg, engine, tmp_path):
    """--phase2-max-y sets phase 2's ceiling apart from phase 1's (-50 here): on hunt.py's
    SCAN_REFERENCE seed over its 40,000-block rect the reference hut (floor -54) is kept at a
    ceiling of -54 or 100 and dropped at -55; at each ceiling the rows and floors equal
    wg_eval_huts' over the phase-1 survivors."""
    seed = 1473884015873122059
    ref = (seed, -987, -1073, -15792, -17168, -54)
    rect = ["--min-region-x", "-79", "--max-region-x", "79", "--min-region-z", "-79", "--max-region-z", "79"]
    cands = engine.seed_check(seeds=[seed], rect=(-79, 79, -79, 79), max_height=-50).candidates
    for ceiling, kept in ((-54, True), (-55, False), (100, True)):
        rows = _scan(wg, tmp_path, "--seed", str(seed), *rect, "--max-height", "-50", "--phase2-max-y",
                     str(ceiling), phase1=False)
        want = exact_rows(engine, cands, ceiling)
        assert rows == want
        assert (ref in want) == kept


def test_self_test_passes(wg, tmp_path):
    """--self-test re-checks the sampled regions through the FP64 noise core: every region of the
    SCAN_REFERENCE seed's 40,000-block rect (24,964 regions, stride 1) and a 20,000-region sample of
    each of 16 seeds of a larger rect."""
    r = subprocess.run([wg.WORKER_PATH, "--seed", "1473884015873122059", "--min-region-x", "-79", "--max-region-x",
                        "79", "--min-region-z", "-79", "--max-region-z", "79", "--max-height", "-50", "--self-test",
                        "--out", "s.csv"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "self-test: checked 24964 sampled regions across 1 seed(s), 0 mismatches -> PASS" in r.stdout
    r = subprocess.run([wg.WORKER_PATH, "--seed-gen", "3", "64", "--min-region-x", "-200", "--max-region-x", "200",
                        "--min-region-z", "-200", "--max-region-z", "200", "--max-height", "100", "--self-test",
                        "--phase1-candidates", "--out", "t.csv"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "self-test: checked 320000 sampled regions across 16 seed(s), 0 mismatches -> PASS" in r.stdout


def _rows(cands):
    return [(int(c["seed"]), int(c["chunk_x"]), int(c["chunk_z"]), int(c["chunk_x"]) * 16, int(c["chunk_z"]) * 16)
            for c in cands]


def _scan(wg, tmp_path, *args, out="q.csv", phase1=True):
    extra = ["--phase1-candidates"] if phase1 else []
    r = subprocess.run([wg.WORKER_PATH, *args, *extra, "--out", out], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return read_csv(tmp_path / out, floor=not phase1)


def test_quad_bases_and_position_gate(wg, port, bind_mod, tmp_path):
    """--quad-bases: the request's seeds are one base's 65,536 high-16-bit variants
    (phase1_scan.cu:79-86); the survivors equal the oracle's over the same expanded seeds, and
    --max-hut-dist keeps those whose reported position is within the distance of the centre."""
    base = 0x0000123456789ABC
    (tmp_path / "bases.txt").write_text(f"999\n{base}\n5\n")
    rect = ["--min-region-x", "-3", "--max-region-x", "3", "--min-region-z", "-3", "--max-region-z", "3",
            "--max-height", "100"]
    seeds = np.array([base | (h << 48) for h in range(65536)], dtype=np.uint64).view(np.int64)
    want, _ = port.scan_seeds(bind_mod.rules("1.19.x~26.1"), 100, (-3, 3, -3, 3), seeds=seeds)
    want_rows = _rows(want)
    assert [(r[1], r[2]) for r in want_rows] == [(8, -22), (2, -84)]
    got = _scan(wg, tmp_path, "--quad-bases", "bases.txt", "--quad-base-offset", "1", "--quad-base-limit", "1",
                *rect)
    assert got == want_rows
    gated = _scan(wg, tmp_path, "--quad-bases", "bases.txt", "--quad-base-offset", "1", "--quad-base-limit", "1",
                  *rect, "--max-hut-dist", "300", "--gate-center-x", "100", "--gate-center-z", "-300")
    assert gated == [r for r in want_rows if (r[3] - 100) ** 2 + (r[4] + 300) ** 2 <= 300 ** 2]
    assert len(gated) == 1


def test_require_all_regions(wg, engine, port, bind_mod, tmp_path):
    """--require-all-regions keeps a seed's candidates only when every region of the rect passes
    the climate gates (phase1_scan.cu:145-181); the kept rows equal the oracle's per-region
    verdicts (codes 0..2 = erosion / temperature / ridge rejections) over the plain scan's seeds."""
    rect = ["--min-region-x", "0", "--max-region-x", "2", "--min-region-z", "0", "--max-region-z", "1",
            "--max-height", "100"]
    gen = ["--seed-gen", "77", str(1 << 24)]
    plain = _scan(wg, tmp_path, *gen, *rect, out="p.csv")
    assert plain == _rows(engine.seed_check(gen=(77, 1 << 24), rect=(0, 2, 0, 1), max_height=100).candidates)
    assert len(plain) == 28
    r = bind_mod.rules("1.19.x~26.1")
    want = [row for row in plain if (port.phase1_rect(row[0], r, 100, (0, 2, 0, 1))[0] > 2).all()]
    assert [(w[1], w[2]) for w in want] == [(12, 18), (8, 11), (19, 1), (50, 1)]
    assert _scan(wg, tmp_path, *gen, *rect, "--require-all-regions", out="a.csv") == want
    both = _scan(wg, tmp_path, *gen, *rect, "--require-all-regions", "--max-hut-dist", "150", "--gate-center-x",
                 "200", "--gate-center-z", "100", out="b.csv")
    assert both == [w for w in want if (w[3] - 200) ** 2 + (w[4] - 100) ** 2 <= 150 ** 2]
    assert len(both) == 2
