"""GPU: the biome map (wg_biome_map, wg_biome_chunks and the biome_map drop-in) against the
reference tool's output (tests/golden/biome_map.npz), byte for byte."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rasters_equal_the_reference(engine, golden):
    d = golden("biome_map.npz")
    for k, meta in enumerate(d["rasters"]):
        seed, ver, x0, z0, w, h, step, ss, y = str(meta).split()
        got = engine.biome_map(int(seed), int(x0), int(z0), int(w), int(h), int(step), int(ss), ver, int(y))
        assert np.array_equal(got, d[f"raster{k}"]), (k, int((got != d[f"raster{k}"]).sum()))


def test_chunks_equal_the_reference(engine, golden):
    d = golden("biome_map.npz")
    seed, ver = str(d["chunks_meta"][0]).split()
    got = engine.biome_chunks(int(seed), d["chunks"][:, 0], d["chunks"][:, 1], ver)
    assert np.array_equal(got, d["chunk_biomes"]), int((got != d["chunk_biomes"]).sum())


def test_cli_bytes(wg, engine, golden):
    d = golden("biome_map.npz")
    seed, ver, x0, z0, w, h, step, ss, y = str(d["rasters"][1]).split()
    r = subprocess.run([wg.BIOME_MAP_PATH, "--seed", seed, "--x0", x0, "--z0", z0, "--w", w, "--h", h, "--step", step,
                        "--ss", ss, "--ver", ver, "--y", y], capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.frombuffer(r.stdout, np.uint8).reshape(int(h), int(w)), d["raster1"])
    seed, ver = str(d["chunks_meta"][0]).split()
    text = "".join(f"{a} {b}\n" for a, b in d["chunks"][:200])
    r = subprocess.run([wg.BIOME_MAP_PATH, "--seed", seed, "--stdin", "--ver", ver], input=text.encode(),
                       capture_output=True, timeout=300)
    assert r.returncode == 0 and r.stdout == d["chunk_biomes"][:200].tobytes()
