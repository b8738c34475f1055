"""Writes the biome-map golden fixtures from the reference's own biome_map tool.

Run from the repository root after `make -C oracle ref REF=<reference root>` (which builds oracle/_ref/biome_map from
engine/tools/mineshaft/biome_map.c and the lysh sources):

    python tests/golden/make_golden_biome.py

biome_map.npz holds, per raster case, the tool's W x H bytes for (seed, --ver, --x0, --z0, --w, --h,
--step, --ss, --y), and for the --stdin case the byte per chunk of a 40 x 40 chunk block around
hunt.py's SCAN_REFERENCE hut (a swamp, so its edges take the real-surface path).
"""
from __future__ import annotations

import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
TOOL = os.path.join(ROOT, "oracle", "_ref", "biome_map")
OUT = os.path.join(ROOT, "tests", "golden", "biome_map.npz")

SCAN_REFERENCE = 1473884015873122059          # hunt.py:86: hut at /tp -15792 -54 -17168
# (seed, version, x0, z0, w, h, step, ss, y)
RASTERS = [(SCAN_REFERENCE, "26.3", -16400, -17800, 64, 64, 24, 1, 63),
           (SCAN_REFERENCE, "1.18.2", -20000, -21000, 48, 40, 96, 3, 63),
           (-5359549684776256167, "1.21.4", 2000000, -1500000, 32, 32, 256, 2, 70),
           (1291329195661654798, "1.20.1", 2137000, 26492600, 40, 24, 32, 4, 56),
           (7, "26.3", -100, -100, 16, 16, 16, 1, 63)]
CHUNKS_SEED, CHUNKS_VER = SCAN_REFERENCE, "26.3"


def main() -> None:
    arrays = {}
    meta = []
    for k, (seed, ver, x0, z0, w, h, step, ss, y) in enumerate(RASTERS):
        r = subprocess.run([TOOL, "--seed", str(seed), "--x0", str(x0), "--z0", str(z0), "--w", str(w), "--h", str(h),
                            "--step", str(step), "--ss", str(ss), "--ver", ver, "--y", str(y)],
                           capture_output=True, check=True)
        assert len(r.stdout) == w * h
        arrays[f"raster{k}"] = np.frombuffer(r.stdout, np.uint8).reshape(h, w)
        meta.append(f"{seed} {ver} {x0} {z0} {w} {h} {step} {ss} {y}")
        print(f"raster {k}: {ver} {w}x{h} step {step} ss {ss}: swamp cells {(arrays[f'raster{k}'] == 6).sum()}")
    cx0, cz0 = -987 - 20, -1073 - 20
    chunks = np.array([(cx0 + i, cz0 + j) for j in range(40) for i in range(40)], dtype=np.int32)
    text = "".join(f"{a} {b}\n" for a, b in chunks)
    r = subprocess.run([TOOL, "--seed", str(CHUNKS_SEED), "--stdin", "--ver", CHUNKS_VER], input=text.encode(),
                       capture_output=True, check=True)
    assert len(r.stdout) == len(chunks)
    arrays["chunks"] = chunks
    arrays["chunk_biomes"] = np.frombuffer(r.stdout, np.uint8).copy()
    print(f"chunks: {len(chunks)}, swamps {(arrays['chunk_biomes'] == 6).sum()}")
    arrays["rasters"] = np.array(meta)
    arrays["chunks_meta"] = np.array([f"{CHUNKS_SEED} {CHUNKS_VER}"])
    np.savez_compressed(OUT, **arrays)


if __name__ == "__main__":
    main()
