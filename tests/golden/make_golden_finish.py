"""Generates tests/golden/finish_rows.npz, the mineshaft finisher's golden values, from the
reference's own finisher tools built here (`make -C oracle ref REF=<reference root>` puts lysh,
mstree, msroom, skyscan and biome_at into oracle/_ref/):

    python tests/golden/make_golden_finish.py

For every row (world seed, hut chunk) it runs exactly what hunt.py's finish_row runs
(hunt.py:277-333): `lysh hut --max-y 100 --phase2-max-y 100 --version 1.19.x~26.1`, `mstree`,
`biome_at --ms --y <room floor>` with and without BIOME_26, `msroom` (MC_SHAPE=79 MC_TRIALS=0, the
tree on stdin) and `skyscan --list` over the 7 x 9 footprint, and keeps the parsed values and
hunt.py's result line.  Rows: hunt.py's REFERENCE, its four TERRAIN_REFERENCE spots with their
known seeds, the 50 located data/finds.tsv huts (read from the reference's data file), start chunks
of the Deep Dive walk fixture under random upper seed bits, and chunks next to starts (no start).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, HERE)
from make_golden_deep import TERRAIN_REFERENCE, read_finds  # noqa: E402

M48 = (1 << 48) - 1
REFERENCE = (3159335117276934358, -1852878, -1380275, 254754461452089, 329, 323)   # hunt.py:83
KIND = {"R": 0, "C": 1, "X": 2, "Y": 3, "S": 4}


def tool(name: str, args: list[str], stdin: str | None = None, env: dict | None = None) -> tuple[int, str]:
    r = subprocess.run([os.path.join(REF, name), *args], input=stdin, capture_output=True, text=True,
                       env=dict(os.environ, **(env or {})), timeout=120)
    return r.returncode, r.stdout


def finish(ws: int, cx: int, cz: int) -> dict:
    """The finisher's values of one row, as finish_row reads them."""
    hx, hz = 16 * cx, 16 * cz
    d = {"ws": ws, "cx": cx, "cz": cz}
    _, out = tool("lysh", ["hut", "--seed", str(ws), "--x", str(hx), "--z", str(hz), "--max-y", "100",
                           "--phase2-max-y", "100", "--version", "1.19.x~26.1"])
    verdict = next((l for l in out.splitlines() if "verdict" in l), "")
    d["verdict_ok"] = int("ACCEPT" in verdict)
    rc, tree = tool("mstree", [str(ws), str(cx), str(cz)])
    d["start"] = int(rc == 0 and bool(tree.strip()))
    d["pieces"] = []
    if not d["start"]:
        return d
    for line in tree.splitlines():
        t = line.split()
        d["pieces"].append([KIND[t[0]]] + [int(v) for v in t[1:10]])
    fl = int(tree.splitlines()[0].split()[2])
    d["floor"] = fl
    for k, env in enumerate((None, {"BIOME_26": "1"})):
        _, bout = tool("biome_at", ["--seed", str(ws), "--cx", str(cx), "--cz", str(cz), "--ms", "--y", str(fl)], env=env)
        d[f"biome{k}"] = int(bout.split()[1])
    _, mout = tool("msroom", ["--seed", str(ws), "--x", str(hx), "--z", str(hz)], stdin=tree,
                   env={"MC_SHAPE": "79", "MC_TRIALS": "0"})
    ex = next(l for l in mout.splitlines() if l.startswith("EXACT")).split()
    d["nat"] = int(ex[5])
    for k, w in enumerate(ex):
        if w in ("top0", "top1", "ng0", "ng1"):
            s, v = ex[k + 1].split("/63=")
            d[f"{w}_sum"], d[w] = int(s), int(v)
        if w == "refused":
            d.setdefault("refused", []).append(int(ex[k + 1]))
    S, u = ws & M48, (ws >> 48) & 0xFFFF
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        f.write("X,u,wx,wz,fw,fd,dx,dz,bound\n%d,%d,%d,%d,7,9,%d,%d,0\n" % (S, u, hx, hz, cx, cz))
        tmp = f.name
    try:
        _, sout = tool("skyscan", ["--list", tmp])
    finally:
        os.remove(tmp)
    w = sout.split()
    get = lambda key: w[w.index(key) + 1]   # noqa: E731
    d["scan_mean"] = float(get("mean"))
    for key, name in (("min", "scan_min"), ("max", "scan_max"), ("le54", "le54"), ("lava", "lava"),
                      ("solid", "solid"), ("NW", "nw"), ("NE", "ne"), ("SW", "sw"), ("SE", "se"),
                      ("above-53", "above53")):
        d[name] = int(get(key))
    return d


def main() -> None:
    rows = [REFERENCE[:3]]
    rows += [(seed, cx, cz) for seed, cx, cz in TERRAIN_REFERENCE]
    rows += [(seed, x // 16, z // 16) for _depth, seed, x, z in read_finds()]
    starts = np.load(os.path.join(HERE, "deep_starts.npz"))
    rng = np.random.default_rng(5)
    walk = np.concatenate([starts["rows0"], starts["rows1"]])
    pick = rng.choice(len(walk), 130, replace=False)
    for r in walk[pick]:
        u = int(rng.integers(0, 1 << 16))
        ws = (u << 48) | (int(r[0]) & M48)
        ws = ws - (1 << 64) if ws >= 1 << 63 else ws
        rows.append((ws, int(r[3]), int(r[4])))
    for ws, cx, cz in rows[:10]:
        rows.append((ws, cx + 1, cz))
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        res = list(ex.map(lambda r: finish(*r), rows))
    n = len(res)
    ints = ["verdict_ok", "start", "floor", "biome0", "biome1", "nat", "top0", "top1", "ng0", "ng1", "top0_sum",
            "top1_sum", "ng0_sum", "ng1_sum", "scan_min", "scan_max", "le54", "lava", "solid", "nw", "ne", "sw",
            "se", "above53"]
    out = {k: np.array([r.get(k, 0) for r in res], dtype=np.int64) for k in ints}
    out["refused"] = np.array([r.get("refused", [0, 0]) for r in res], dtype=np.int64).reshape(n, 2)
    out["scan_mean"] = np.array([r.get("scan_mean", 0.0) for r in res])
    out["ws"] = np.array([r["ws"] for r in res], dtype=np.int64)
    out["cx"] = np.array([r["cx"] for r in res], dtype=np.int32)
    out["cz"] = np.array([r["cz"] for r in res], dtype=np.int32)
    out["n_pieces"] = np.array([len(r["pieces"]) for r in res], dtype=np.int64)
    out["pieces"] = np.array([p for r in res for p in r["pieces"]], dtype=np.int64).reshape(-1, 10)
    np.savez_compressed(os.path.join(HERE, "finish_rows.npz"), **out)
    print(f"{n} rows, {int(out['start'].sum())} starts, {int(out['verdict_ok'].sum())} accepted, "
          f"{len(out['pieces'])} pieces; REFERENCE top1 {int(out['top1'][0])}")


if __name__ == "__main__":
    main()
