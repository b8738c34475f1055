"""GPU: the Deep Dive entry points against the reference's own values.

wg_deep_starts (the region walk) must return exactly the rows of the reference's room walker
(tests/golden/deep_starts.npz) with the oracle's carver state; wg_deep_spots (the terrain stage
over the 65,536 upper-bit variants) must keep exactly the variants lysh's phase 1 keeps
(tests/golden/deep_spots.npz) — for hunt.py's TERRAIN_REFERENCE spots, the known seeds.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_deep_starts_match_reference(engine, port):
    d = np.load(os.path.join(GOLDEN, "deep_starts.npz"))
    for k, rect in enumerate(d["rects"]):
        got = engine.deep_starts(s48=d["s48"], rect=tuple(int(v) for v in rect))
        rows = np.stack([got["s48"], got["rx"], got["rz"], got["chunk_x"], got["chunk_z"]], 1).astype(np.int64)
        assert np.array_equal(rows, d[f"rows{k}"]), k
        want = port.deep_starts(d["s48"], tuple(int(v) for v in rect))
        assert np.array_equal(got["carver"], want[:, 5]), k


def test_deep_starts_generator_and_capacity(engine, port):
    got = engine.deep_starts(base=12345, count=6, rect=(-300, 300, -200, 200))
    want = port.deep_starts([12345 + i for i in range(6)], (-300, 300, -200, 200), cap=1 << 15)
    assert len(got) == len(want) > 4096   # exercises the capacity retry
    assert np.array_equal(np.stack([got["s48"], got["rx"], got["rz"]], 1), want[:, :3])


def test_deep_starts_first_cap_in_order(engine, wg):
    """With room for fewer hits than there are, the call writes the first ones of the
    (seed_index, rz, rx) order and reports the total (include/witchgpu.h)."""
    import ctypes as C
    full = engine.deep_starts(base=777, count=3, rect=(-100, 100, -100, 100))
    assert len(full) > 300
    for cap in (1, len(full) // 3, len(full) - 1):
        out = np.zeros(cap, wg.DEEP_START_DTYPE)
        found = C.c_uint64()
        rc = wg.library().wg_deep_starts(engine._h, None, 777, 3, -100, 100, -100, 100, out.ctypes.data, cap,
                                         C.byref(found))
        assert rc == 0 and found.value == len(full)
        assert np.array_equal(out, full[:cap]), cap


def test_deep_starts_several_passes(engine):
    """A walk of more than 2^24 (seed, row, strip) tasks runs in passes whose outputs continue one
    another: it equals the same seeds walked in two calls."""
    rect = (-2048, 2048, -2048, 2048)   # 4,096 rows x 64 strips per seed: 65 seeds = 2 passes
    whole = engine.deep_starts(base=4242, count=65, rect=rect)
    a = engine.deep_starts(base=4242, count=33, rect=rect)
    b = engine.deep_starts(base=4242 + 33, count=32, rect=rect)
    b = b.copy()
    b["seed_index"] += 33
    assert len(whole) == len(a) + len(b) > 1_000_000
    assert np.array_equal(whole, np.concatenate([a, b]))


def test_deep_spots_match_reference(engine):
    d = np.load(os.path.join(GOLDEN, "deep_spots.npz"))
    surv, bad = engine.deep_spots(d["s48"], d["chunk_x"], d["chunk_z"], max_height=int(d["max_height"]))
    assert bad == int((d["start"] == 0).sum())
    off = np.concatenate([[0], np.cumsum(d["counts"])])
    want = [(i << 16) | int(u) for i in range(len(d["s48"])) for u in d["passed"][off[i]:off[i + 1]]]
    assert surv["seed_index"].tolist() == want
    for row in surv:
        i, u = int(row["seed_index"]) >> 16, int(row["seed_index"]) & 0xFFFF
        assert (int(row["seed"]) & ((1 << 64) - 1)) == (u << 48) | int(d["s48"][i])
        assert (row["chunk_x"], row["chunk_z"]) == (d["chunk_x"][i], d["chunk_z"][i])
    # every known find (hunt.py's TERRAIN_REFERENCE and the 50 located data/finds.tsv huts) survives
    got = set(int(s) for s in surv["seed"])
    for i, seed in enumerate(d["seed"]):
        if int(seed):
            assert int(seed) in got, (i, int(seed))
