"""GPU: the hut_lookup worker binary speaks the reference Deep Dive engine's command-line contract
(hut_lookup_v4 --solve-only --solve5 --plan ... --dump-hits, and --spots ... --out), as hunt.py runs
it (hunt.py:947-957), and gives the reference's answers (tests/golden/deep_solve.npz,
tests/golden/deep_spots.npz)."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M48 = (1 << 48) - 1


def test_solver_command(wg, engine, golden, tmp_path):
    d = golden("deep_solve.npz")
    lay, rgx, rgz, tier, first, count = (int(v) for v in d["cases"][0])
    (tmp_path / "cat.txt").write_text(f"{lay} 331 331\n")
    (tmp_path / "plan.txt").write_text(f"{lay} {rgx}{rgz} odd 1 7.7e11 1 1\n")
    hits = tmp_path / "hits.csv"
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--catalog", "cat.txt", "--solve-only", "--solve5", "--plan", "plan.txt",
                        "--fused-blk", "64", "--fused-grid", "0", "--fused-gpb", "32", "--fused-slots", "2",
                        "--fused-threads", "2", "--regime", "22", "--first-index", str(first), "--count", str(count),
                        "--task-batch", "4096", "--quiet", "--dump-hits", str(hits), "--out", "dummy.csv"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "solve:" in r.stdout
    rows = sorted((int(p[0]), int(p[1]), int(p[2])) for p in (l.split(",") for l in hits.read_text().split())
                  if len(p) == 5 and int(p[3]) == lay and p[4] == "1")
    assert rows == sorted((int(h[0]) & M48, int(h[1]), int(h[2])) for h in d["hits0"])


def test_terrain_command(wg, engine, golden, tmp_path):
    d = golden("deep_spots.npz")
    starts = [i for i in range(len(d["s48"])) if d["start"][i]]
    lines = [f"{int(d['s48'][i])} {int(d['chunk_x'][i])} {int(d['chunk_z'][i])}" for i in starts]
    (tmp_path / "spots.txt").write_text("\n".join(lines) + "\n")
    (tmp_path / "cat.txt").write_text("231564844655014 331 331\n")
    out = tmp_path / "surv.csv"
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--catalog", "cat.txt", "--spots", "spots.txt", "--batch", "64",
                        "--ero-split", "--ero-t1", "0.5", "--ero-c0", "0.1", "--ero-t3", "0.5", "--ero-c1", "0.1",
                        "--max-height", "-54", "--quiet", "--out", str(out)],
                       capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    text = out.read_text().split("\n")
    assert text[0] == "seed,chunkX,chunkZ,layoutX,airHi,airLo"
    got = sorted((int(p[0]) & 0xFFFFFFFFFFFFFFFF, int(p[1]), int(p[2])) for p in (l.split(",") for l in text[1:] if l))
    want = []
    at = np.concatenate([[0], np.cumsum(d["counts"])])
    for i in starts:
        for u in d["passed"][at[i]:at[i + 1]]:
            want.append(((int(u) << 48) | (int(d["s48"][i]) & M48), int(d["chunk_x"][i]), int(d["chunk_z"][i])))
    assert got == sorted(want)
    # a chunk that is not a mineshaft start: reported, exit 1
    bad = [i for i in range(len(d["s48"])) if not d["start"][i]]
    if bad:
        i = bad[0]
        (tmp_path / "bad.txt").write_text(f"{int(d['s48'][i])} {int(d['chunk_x'][i])} {int(d['chunk_z'][i])}\n")
        r = subprocess.run([wg.HUT_LOOKUP_PATH, "--catalog", "cat.txt", "--spots", "bad.txt", "--out", "b.csv"],
                           capture_output=True, text=True, cwd=tmp_path, timeout=600)
        assert r.returncode == 1 and "not" in r.stderr


def test_finish_command(wg, tmp_path):
    """hut_lookup --finish over the finisher fixture's rows prints, for every row hunt.py's
    finish_row accepts, the same line finish_row builds from the reference tools' outputs
    (hunt.py:277-333), and nothing for the others; hunt.py's selftest condition holds for REFERENCE."""
    import os
    fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "finish_rows.npz"))
    layout, hi, lo = ["0"] * len(fx["ws"]), ["0"] * len(fx["ws"]), ["0"] * len(fx["ws"])
    layout[0], hi[0], lo[0] = "254754461452089", "329", "323"   # hunt.py:83
    with open(tmp_path / "rows.csv", "w") as f:
        f.write("seed,chunkX,chunkZ,layoutX,airHi,airLo\n")
        for i in range(len(fx["ws"])):
            f.write(f"{int(fx['ws'][i])},{int(fx['cx'][i])},{int(fx['cz'][i])},{layout[i]},{hi[i]},{lo[i]}\n")
    r = subprocess.run([wg.HUT_LOOKUP_PATH, "--finish", "rows.csv"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    want = []
    for i in range(len(fx["ws"])):
        if not (fx["verdict_ok"][i] and fx["start"][i]) or (fx["biome0"][i] == 183 and fx["biome1"][i] == 183):
            continue
        r1 = int(fx["top1"][i])
        want.append("%4d  terrain %4s  refused %2s  if-none-refused %4s  NW %4s  max %4s  lava %4s  air %s/%s  "
                    "biome %s  layout %s  seed %s  /tp %d %d %d"
                    % (r1, fx["nat"][i], fx["refused"][i][0], fx["ng1"][i], fx["nw"][i], fx["scan_max"][i],
                       fx["lava"][i], hi[i], lo[i], fx["biome0"][i], layout[i], int(fx["ws"][i]),
                       16 * int(fx["cx"][i]), r1, 16 * int(fx["cz"][i])))
    assert r.stdout.splitlines() == want
    assert len(want) > 50
    assert int(want[0].split()[0]) <= -58 and "/tp -29646048 -58 -22084400" in want[0]
