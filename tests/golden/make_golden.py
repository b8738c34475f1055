"""Generates the golden fixtures in this folder from the reference's own lysh.

Run from the repository root after `make -C oracle ref REF=<reference root>` (which compiles lysh from the
reference sources into oracle/_ref/):

    python tests/golden/make_golden.py

Every number written here comes from liblysh_ref.so, i.e. the reference implementation;
the tests compare both the C restatement (oracle/) and the CUDA engine against them.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import bind  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
RECT9 = (-4, 5, -4, 5)

# Option sets exercised: (version, preset, phase-1 maxHeight)
VARIANTS = [("1.19.x~26.1", "NORMAL", -50), ("26.2", "NORMAL", -40), ("1.18.2", "NORMAL", -50),
            ("1.19.x~26.1", "LARGE_BIOMES", -50), ("1.19.x~26.1", "SINGLE_BIOME", -50),
            ("1.19.x~26.1", "NORMAL", 100), ("1.19.x~26.1", "NORMAL", -45)]

NOISES = ["minecraft:erosion", "minecraft:temperature", "minecraft:ridge", "minecraft:continentalness",
          "minecraft:erosion_large", "minecraft:temperature_large", "minecraft:continentalness_large",
          "minecraft:cave_entrance", "minecraft:spaghetti_3d_rarity", "minecraft:spaghetti_3d_thickness",
          "minecraft:spaghetti_3d_1", "minecraft:spaghetti_3d_2", "minecraft:spaghetti_roughness_modulator",
          "minecraft:spaghetti_roughness", "minecraft:cave_layer", "minecraft:cave_cheese",
          "minecraft:aquifer_fluid_level_floodedness"]


def splitmix64(x: int) -> int:
    m = 0xFFFFFFFFFFFFFFFF
    x = (x + 0x9E3779B97F4A7C15) & m
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def main() -> None:
    ref = bind.Ref()
    r = bind.rules("1.19.x~26.1")

    # 1. config 1: 4,096 seeds splitmix64(1 + i) x 9x9 regions, maxHeight -50
    seeds = np.array([splitmix64(1 + i) for i in range(4096)], dtype=np.uint64)
    codes = np.zeros((4096, 81), np.int8)
    tiers = np.zeros((4096, 81), np.int8)
    for i, s in enumerate(seeds):
        c, t, _, _ = ref.phase1_rect(int(s), r, -50, RECT9)
        codes[i], tiers[i] = c, t
    np.savez_compressed(os.path.join(OUT, "c1_phase1.npz"), seeds=seeds, codes=codes, tiers=tiers)

    # 2. rule variants on 64 seeds
    var = {}
    for k, (version, preset, mh) in enumerate(VARIANTS):
        rv = bind.rules(version, preset)
        cs = np.zeros((64, 81), np.int8)
        ts = np.zeros((64, 81), np.int8)
        for i in range(64):
            c, t, _, _ = ref.phase1_rect(int(seeds[i]), rv, mh, RECT9)
            cs[i], ts[i] = c, t
        var[f"codes_{k}"] = cs
        var[f"tiers_{k}"] = ts
    np.savez_compressed(os.path.join(OUT, "variants.npz"), seeds=seeds[:64], **var)

    # 3. the 38 raw probe doubles at 48 (seed, hut) points under three maxHeights
    rng = np.random.default_rng(20261203)
    pts, vals = [], []
    for _ in range(16):
        s = int(rng.integers(0, 2 ** 64, dtype=np.uint64))
        hx = int(rng.integers(-1_800_000, 1_800_000)) * 16
        hz = int(rng.integers(-1_800_000, 1_800_000)) * 16
        for mh in (-50, -40, 100):
            pts.append((s, hx, hz, mh))
            vals.append(ref.probe(s, r, hx, hz, mh))
    np.savez_compressed(os.path.join(OUT, "probes.npz"), seeds=np.array([p[0] for p in pts], np.uint64),
                        hx=np.array([p[1] for p in pts], np.int32), hz=np.array([p[2] for p in pts], np.int32),
                        mh=np.array([p[3] for p in pts], np.int32), values=np.array(vals))

    # 4. constructed noise samplers: amplitude / lacunarity / persistence, origins, perm digests
    tables = {}
    for s in (0, 1473884015873122059, 0xFFFFFFFFFFFFFFFF):
        for name in NOISES:
            h, pr, org, pm = ref.noise_dump(s, name)
            tables[f"{s}|{name}"] = {"head": [float(x).hex() for x in h], "present": pr.tolist(),
                                     "origin": [float(x).hex() for x in org],
                                     "perm_sha256": hashlib.sha256(pm.tobytes()).hexdigest()}
    with open(os.path.join(OUT, "noise_tables.json"), "w") as f:
        json.dump(tables, f, indent=0, sort_keys=True)

    # 5. known answers from the reference's own tests / docs, restated as phase-1 survivor sets
    known = {}
    # hunt.py:86 SCAN_REFERENCE and tools/test_hunt.py:264-277: found in a 40,000-block area
    # (regions [-79, 79)), not in a 5,000-block one ([-10, 10)).
    for label, rect in (("scan_reference_40000", (-79, 79, -79, 79)), ("scan_reference_5000", (-10, 10, -10, 10))):
        c, _, cx, cz = ref.phase1_rect(1473884015873122059, r, -50, rect)
        idx = np.nonzero(c == 10)[0]
        known[label] = {"seed": 1473884015873122059, "rect": rect,
                        "hist": np.bincount(c, minlength=11).tolist(),
                        "survivors": [[int(cx[i]), int(cz[i])] for i in idx]}
    # docs/HUNT54.txt:18-19, docs/VERIFIED.txt:9-13: seed 1291329195661654798 -> /tp 2137600 -54 26493184
    rect = (4170, 4180, 51740, 51750)
    c, _, cx, cz = ref.phase1_rect(1291329195661654798, r, -50, rect)
    idx = np.nonzero(c == 10)[0]
    known["verified_54"] = {"seed": 1291329195661654798, "rect": rect,
                            "hist": np.bincount(c, minlength=11).tolist(),
                            "survivors": [[int(cx[i]), int(cz[i])] for i in idx]}
    # lysh hut on those two huts (phase 2, kept for the phase-2 parity work)
    for label, seed, hx, hz in (("hut_scan_reference", 1473884015873122059, -15792, -17168),
                                ("hut_verified_54", 1291329195661654798, 2137600, 26493184)):
        mc, pre, tree = ref.version("1.19.x~26.1")
        ctx = ref.lib.refh_ctx_new(seed, mc, pre, 0, 0, tree, -50)
        out = np.zeros(24, np.int64)
        ref.lib.refh_ctx_eval(ctx, hx, hz, -50, out.ctypes.data)
        ref.lib.refh_ctx_free(ctx)
        known[label] = {"seed": seed, "hut": [hx, hz], "eval": out.tolist()}
    # hut placement + orientation on a grid of seeds/regions (integer stage)
    place = []
    for k in range(64):
        s = splitmix64(1000 + k)
        rx, rz = int(rng.integers(-58594, 58594)), int(rng.integers(-58594, 58594))
        cxz = np.zeros(2, np.int32)
        ref.lib.refh_hut_in_region(s, rx, rz, 0, cxz[0:].ctypes.data, cxz[1:].ctypes.data)
        d = ref.lib.refh_hut_orientation(s, int(cxz[0]) * 16, int(cxz[1]) * 16)
        place.append([str(s), rx, rz, int(cxz[0]), int(cxz[1]), int(d)])
    known["placement"] = place
    with open(os.path.join(OUT, "known_answers.json"), "w") as f:
        json.dump(known, f, indent=1)

    # 6. config 2 sample: the first 65,536 seeds of splitmix64(2 + i) -> survivors and funnel
    hist = np.zeros(11, np.int64)
    surv = []
    for i in range(65536):
        s = splitmix64(2 + i)
        c, _, cx, cz = ref.phase1_rect(s, r, -50, RECT9)
        hist += np.bincount(c, minlength=11)
        for k in np.nonzero(c == 10)[0]:
            surv.append((i, s - (1 << 64) if s >= (1 << 63) else s,
                         int(k % 9) - 4, int(k // 9) - 4, int(cx[k]), int(cz[k])))
    surv = np.array(surv, dtype=bind.CANDIDATE_DTYPE)
    np.savez_compressed(os.path.join(OUT, "c2_sample.npz"), survivors=surv, hist=hist)

    # 7. config 2, first 2^22 seeds and all 2^24 seeds: every phase-1 survivor (lysh's own threaded
    # scan finds the seeds, lysh_phase1_rect gives their regions and chunks)
    for n, name in ((1 << 22, "c2_4m_survivors.npz"), (1 << 24, "c2_full_survivors.npz")):
        c2_survivors(ref, r, n, name)
    print("golden fixtures written to", OUT)


def c2_survivors(ref, r, n, name):
    idx = np.arange(n, dtype=np.uint64) + np.uint64(2)
    with np.errstate(over="ignore"):
        z = idx + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        seeds2 = z ^ (z >> np.uint64(31))
    _, acc = ref.phase1_seeds(seeds2, r, -50, RECT9)
    surv = []
    for i in np.nonzero(acc)[0]:
        s = int(seeds2[i])
        c, _, cx, cz = ref.phase1_rect(s, r, -50, RECT9)
        for k in np.nonzero(c == 10)[0]:
            surv.append((int(i), s - (1 << 64) if s >= (1 << 63) else s,
                         int(k % 9) - 4, int(k // 9) - 4, int(cx[k]), int(cz[k])))
    np.savez_compressed(os.path.join(OUT, name), survivors=np.array(surv, dtype=bind.CANDIDATE_DTYPE), n_seeds=n)


if __name__ == "__main__":
    main()
