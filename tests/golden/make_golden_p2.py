"""Generates the phase-2 golden fixtures in this folder from the reference's own lysh.

Run from the repository root after `make -C oracle ref REF=<reference root>` (lysh compiled from the reference
sources into oracle/_ref/):

    python tests/golden/make_golden_p2.py

Every value written comes from liblysh_ref.so through oracle/ref_harness.c (lysh_eval_hut,
lysh_grade_scan and the phase-2 probes), i.e. from the reference implementation:

  p2_probes.npz  per seed and probe kind (the kinds of wg_p2_probe): block points and lysh's
                 value there (blended noise, raw and interpolated density, column tops, terrain
                 info, computeFluid, block states, surface heights before / after carvers)
  p2_huts.npz    lysh_eval_hut on forced hut positions: the 81 region huts of the first config-1
                 seeds (hunt.py's version), a few seeds under other versions / presets, the
                 185 phase-1 survivors of config 2, the SCAN_REFERENCE hut and the 50 located
                 data/finds.tsv huts (the reference's data file, read at generation time)
  p2_grade.json  lysh_grade_scan of the SCAN_REFERENCE seed over its 40,000-block rect
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import bind  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SCAN_REFERENCE = 1473884015873122059
RECT9 = (-4, 5, -4, 5)
MAX_Y = -50


def splitmix64(x: int) -> int:
    m = 0xFFFFFFFFFFFFFFFF
    x = (x + 0x9E3779B97F4A7C15) & m
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def opts_of(ref: bind.Ref, version: str, preset: str = "NORMAL") -> list[int]:
    """wg_opts field order: mc_1_18_2, single_biome, pre_26_2, large_biomes, biome_tree."""
    mc, pre, tree = ref.version(version)
    return [mc, int(preset == "SINGLE_BIOME"), pre, int(preset == "LARGE_BIOMES"), tree]


def rules_of(o: list[int]) -> dict:
    return {"mc_1_18_2": o[0], "single_biome": o[1], "pre_26_2": o[2], "large_biomes": o[3]}


def probes(ref: bind.Ref) -> None:
    rng = np.random.default_rng(7)
    seeds = [SCAN_REFERENCE, splitmix64(1)]
    o = opts_of(ref, "1.19.x~26.1")
    arrays = {"seeds": np.array(seeds, dtype=np.uint64), "opts": np.array(o, np.int32)}
    for si, seed in enumerate(seeds):
        with ref.ctx(seed, rules_of(o), -50, o[4]) as ctx:
            for kind in range(10):   # per-point kinds: scattered over +-3000 blocks
                n = 96 if kind == 9 else 192
                pts = np.stack([rng.integers(-3000, 3000, n), rng.integers(-64, 320, n),
                                rng.integers(-3000, 3000, n)], axis=1).astype(np.int32)
                arrays[f"s{si}_k{kind}_pts"] = pts
                arrays[f"s{si}_k{kind}_vals"] = ctx.probe(kind, pts)
            # per-chunk kinds: points inside a few chunks (the SCAN_REFERENCE hut's chunk first)
            chunks = [(-987, -1073)] + [tuple(int(v) for v in rng.integers(-150, 150, 2)) for _ in range(2)]
            for kind in (10, 11, 12, 13):
                rows = []
                for cx, cz in chunks:
                    m = 12 if kind >= 12 else 40
                    x = cx * 16 + rng.integers(0, 16, m)
                    z = cz * 16 + rng.integers(0, 16, m)
                    y = rng.integers(-64, 320, m)
                    rows.append(np.stack([x, y, z], axis=1))
                pts = np.concatenate(rows).astype(np.int32)
                arrays[f"s{si}_k{kind}_pts"] = pts
                arrays[f"s{si}_k{kind}_vals"] = ctx.probe(kind, pts)
    np.savez_compressed(os.path.join(OUT, "p2_probes.npz"), **arrays)


def huts(ref: bind.Ref) -> None:
    rows = []   # (set, seed, hut_x, hut_z, opts..., eval fields...)

    def add(tag: int, seed: int, o: list[int], hxz: list[tuple[int, int]]) -> None:
        with ref.ctx(seed, rules_of(o), -50, o[4]) as ctx:
            for hx, hz in hxz:
                e = ctx.eval_hut(hx, hz, MAX_Y)
                signed = seed - (1 << 64) if seed >= (1 << 63) else seed
                rows.append([tag, signed, hx, hz] + o + [e[f] for f in bind.EVAL_FIELDS])

    def region_huts(seed: int, o: list[int]) -> list[tuple[int, int]]:
        _, _, cx, cz = ref.phase1_rect(seed, rules_of(o), -50, RECT9, tree=o[4])
        return [(int(a) * 16, int(b) * 16) for a, b in zip(cx, cz)]

    # set 0: the 81 region huts of the first 12 config-1 seeds, hunt.py's version
    o = opts_of(ref, "1.19.x~26.1")
    for i in range(12):
        s = splitmix64(1 + i)
        add(0, s, o, region_huts(s, o))
    # set 1: other versions / presets, 2 seeds each
    for ver, preset in (("26.2", "NORMAL"), ("1.18.2", "NORMAL"), ("1.19.x~26.1", "LARGE_BIOMES"),
                        ("1.21", "NORMAL")):
        ov = opts_of(ref, ver, preset)
        for i in range(2):
            s = splitmix64(101 + i)
            add(1, s, ov, region_huts(s, ov))
    # set 2: the config-2 phase-1 survivors
    surv = np.load(os.path.join(OUT, "c2_full_survivors.npz"))["survivors"]
    by_seed: dict[int, list[tuple[int, int]]] = {}
    for c in surv:
        by_seed.setdefault(int(c["seed"]), []).append((int(c["chunk_x"]) * 16, int(c["chunk_z"]) * 16))
    for s, hxz in by_seed.items():
        add(2, s, o, hxz)
    # set 3: the SCAN_REFERENCE hut
    add(3, SCAN_REFERENCE, o, [(-987 * 16, -1073 * 16)])
    # set 4: every located data/finds.tsv hut (real deep huts: biome-OK and dry; their plain-terrain
    # floor, before the mineshaft room the finisher adds, decides the verdict at the ceiling)
    from make_golden_deep import read_finds
    for _depth, seed, x, z in read_finds():
        add(4, seed & 0xFFFFFFFFFFFFFFFF, o, [((x // 16) * 16, (z // 16) * 16)])
    cols = ["set", "seed", "hut_x", "hut_z", "mc_1_18_2", "single_biome", "pre_26_2", "large_biomes",
            "biome_tree"] + list(bind.EVAL_FIELDS)
    out = {c: np.array([int(r[i]) for r in rows], dtype=np.int64) for i, c in enumerate(cols)}
    out["columns"] = np.array(cols)
    np.savez_compressed(os.path.join(OUT, "p2_huts.npz"), **out)


def grade(ref: bind.Ref) -> None:
    o = opts_of(ref, "1.19.x~26.1")
    rect = (-79, 79, -79, 79)
    hits, st = ref.grade_scan(SCAN_REFERENCE, rules_of(o), -50, rect, MAX_Y, tree=o[4])
    with open(os.path.join(OUT, "p2_grade.json"), "w") as f:
        json.dump({"seed": SCAN_REFERENCE, "rect": rect, "max_height": -50, "max_y": MAX_Y, "opts": o,
                   "hits": hits.tolist(), "stats": [int(v) for v in st]}, f, indent=1)


def main() -> None:
    ref = bind.Ref()
    probes(ref)
    huts(ref)
    grade(ref)


if __name__ == "__main__":
    main()
