"""CPU: the biome-map fixtures are the reference tool's output (re-run it when it is built here),
and the biome_map drop-in refuses bad command lines like the reference (exit 2)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(ROOT, "oracle", "_ref", "biome_map")


def test_fixture_is_the_reference_output(golden):
    if not os.path.exists(TOOL):
        pytest.skip("oracle/_ref/biome_map not built (needs the reference sources)")
    d = golden("biome_map.npz")
    for k, meta in enumerate(d["rasters"]):
        seed, ver, x0, z0, w, h, step, ss, y = str(meta).split()
        r = subprocess.run([TOOL, "--seed", seed, "--x0", x0, "--z0", z0, "--w", w, "--h", h, "--step", step,
                            "--ss", ss, "--ver", ver, "--y", y], capture_output=True, check=True)
        assert np.array_equal(np.frombuffer(r.stdout, np.uint8).reshape(int(h), int(w)), d[f"raster{k}"])


@pytest.mark.parametrize("args", [["--seed", "1"], ["--seed", "1", "--x0", "0", "--z0", "0", "--w", "5000", "--h", "1"],
                                  ["--seed", "1", "--stdin", "--ss", "5"], ["--seed", "1", "--stdin", "--ver", "1.17"],
                                  ["--bogus"]])
def test_biome_map_cli_usage(wg, args):
    r = subprocess.run([wg.BIOME_MAP_PATH] + args, capture_output=True, text=True, input="")
    assert r.returncode == 2
